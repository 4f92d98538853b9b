#!/usr/bin/env python
"""Encoded macroblocks per second of the B200 H.261 core.

One step = one frame-step of the workload: the next picture of every stream
of the batch, encoded in one launch of the core (motion search, mode
decision, motion compensation with the loop filter, DCT, denoise,
quantisation, dequantisation, IDCT, reconstruction).  Workload: ``batch64``
(40 QCIF + 24 CIF streams, QUANT 4..24, seeded synthetic content; see
h261enc_cuda_b200/workloads.py).

  value   device throughput: pictures already in HBM, L2 flushed (256 MiB
          write) before every timed step, the step kernel timed with CUDA
          events on the engine's stream;
  e2e     the same through the public API with host buffers: every step
          copies its pictures from host memory into the pinned arena, moves
          them to the device, encodes, and reads the compact results back;
  single_stream  the same streams one at a time (one picture per step,
          synchronous), the plain single-stream path;
  latency_ms     per-picture latency (submit -> results on the host).

``--impl reference`` times the CPU restatement of the reference's device
path (oracle/) on all host cores instead.  Under torchrun every rank encodes
its own batch (weak scaling, no collective on the data path); rank 0 prints
one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CLIP_LEN = 24
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "step_kernel_batch64.md")
# algorithmic bytes per MB: source 384 + reference 384 + reconstruction 384
# + levels 384 (int8) + MB record 16 + work item 4
ALG_BYTES_PER_MB = 384 + 384 + 384 + 384 + 16 + 4
# reference-mode search: 121 + 49 candidates x 256 absolute differences
SAD_PER_MB = 170 * 256


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# --------------------------------------------------------------- helpers

class ClockSampler:
    """nvidia-smi samples (200 ms) while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").strip().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                mx = float(p[1])
            except ValueError:
                continue
            for n, v in zip(names, p[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    try:
        v = json.load(open(MEASURED_PEAKS))["hbm_gbs"]
        return float(v), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic_per_mb():
    """DRAM bytes per MB of the step kernel from the committed ncu summary."""
    try:
        for line in open(PROFILE_SUMMARY):
            if line.startswith("dram_bytes_per_mb:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=datetime.timedelta(seconds=120))
    return world, rank, local, dist


# ------------------------------------------------------------ CPU baseline

def cpu_baseline(streams, frames_per_stream: int, threads: int):
    """The oracle (C restatement of the reference's device path) over a
    bounded sample: each task encodes one stream's first pictures."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from h261enc_cuda_b200 import workloads
    clips = [workloads.make_clip(s, frames_per_stream) for s in streams]

    def task(i):
        s = streams[i]
        O.encode_sequence(clips[i], s.width, s.height, s.quant)
        return s.num_mb * frames_per_stream

    O.lib()
    t = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        mbs = sum(ex.map(task, range(len(streams))))
    el = time.perf_counter() - t
    return mbs, el


def reference_arm(args, world, rank):
    from h261enc_cuda_b200 import workloads
    if rank != 0:
        return
    streams = workloads.WORKLOADS[args.workload]()
    threads = os.cpu_count() or 1
    frames = 3
    for _ in range(args.warmup):
        cpu_baseline(streams[:threads], 2, threads)
    times, total = [], 0
    for _ in range(args.steps):
        mbs, el = cpu_baseline(streams, frames, threads)
        times.append(el)
        total += mbs
    value = total / sum(times)
    sample = f"{len(streams)} streams x {frames} pictures per step (oracle, C, -O2)"
    line = {"impl": "reference", "metric": "encoded MB/s", "value": value, "unit": "MB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": args.workload, "streams": len(streams), "mb_per_step": total // args.steps},
            "cpu_baseline": {"value": value, "unit": "MB/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- ours

def device_clips(streams, clip_len, device):
    """Clips of every stream in HBM: planes 256-byte aligned per picture."""
    import torch
    from h261enc_cuda_b200 import workloads
    pools = []
    for s in streams:
        w, h = s.width, s.height
        ny, nc = w * h, w * h // 4
        off_cb = (ny + 255) // 256 * 256
        off_cr = off_cb + (nc + 255) // 256 * 256
        stride = off_cr + (nc + 255) // 256 * 256
        host = workloads.make_clip(s, clip_len)
        buf = np.zeros((clip_len, stride), np.uint8)
        buf[:, :ny] = host[:, :ny]
        buf[:, off_cb:off_cb + nc] = host[:, ny:ny + nc]
        buf[:, off_cr:off_cr + nc] = host[:, ny + nc:]
        t = torch.from_numpy(buf).to(f"cuda:{device}")
        base = t.data_ptr()
        pools.append((t, host, [(base + i * stride, base + i * stride + off_cb, base + i * stride + off_cr)
                                for i in range(clip_len)]))
    return pools


class Runner:
    """Keeps the workload's slots full: a stream that reaches its length is
    closed and a new session (same geometry and QUANT) takes the slot."""

    def __init__(self, engine, streams):
        self.e, self.streams = engine, streams
        self.sids = [engine.open(s.width, s.height, s.quant) for s in streams]
        self.pos = [0] * len(streams)

    def queue(self, pools, on_device: bool):
        from h261enc_cuda_b200 import workloads
        for k, s in enumerate(self.streams):
            if self.pos[k] >= s.length:
                self.e.close(self.sids[k])
                self.sids[k] = self.e.open(s.width, s.height, s.quant)
                self.pos[k] = 0
            i = workloads.clip_index(self.pos[k], CLIP_LEN)
            if on_device:
                self.e.submit_device(self.sids[k], *pools[k][2][i])
            else:
                self.e.submit_frame(self.sids[k], pools[k][1][i])
            self.pos[k] += 1


def ours(args, world, rank, local, dist):
    import torch
    from h261enc_cuda_b200 import workloads
    from h261enc_cuda_b200.engine import Engine, sad_peak

    torch.cuda.set_device(local)
    streams = workloads.WORKLOADS[args.workload](rank=rank)
    mb_per_step = sum(s.num_mb for s in streams)
    pools = device_clips(streams, CLIP_LEN, local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    peak_sad = sad_peak(local)

    eng = Engine(device=local, max_sessions=4 * len(streams))
    run = Runner(eng, streams)
    # warm-up (includes the launch-shape tuning steps)
    for _ in range(max(args.warmup, 8)):
        run.queue(pools, True)
        eng.step()
        eng.sync()

    # ---- value: device-resident pictures, L2 flushed, kernel events
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    kernel_ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            run.queue(pools, True)
            eng.step()
            kernel_ms.append(eng.last_kernel_ms())
        eng.sync()
    torch.cuda.synchronize()
    total_ms = float(sum(kernel_ms))
    if dist:
        t = torch.tensor([total_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = mb_per_step * args.steps * world / (total_ms * 1e-3)

    # ---- e2e: host pictures through the public API, results read back
    h2d = sum(s.width * s.height * 3 // 2 for s in streams)
    d2h = sum(s.num_mb * (16 + 384) for s in streams)
    lat = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ts = time.perf_counter()
        run.queue(pools, False)
        eng.step()
        eng.sync()
        chk = 0
        for sid in run.sids[:1]:
            chk += int(eng.result(sid, copy=False).mbs["cost"].sum())
        lat.append((time.perf_counter() - ts) * 1e3)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = mb_per_step * args.steps * world / e2e_s
    eng.destroy()

    # ---- single stream: the same streams one at a time, one picture per step
    single_lat, single_mbs = [], 0
    eng1 = Engine(device=local, max_sessions=8, warps_per_cta=4)
    per_stream = 3
    t0 = time.perf_counter()
    for k, s in enumerate(streams):
        sid = eng1.open(s.width, s.height, s.quant)
        for i in range(per_stream):
            ts = time.perf_counter()
            eng1.submit_frame(sid, pools[k][1][i])
            eng1.step()
            eng1.sync()
            eng1.result(sid, copy=False)
            single_lat.append((time.perf_counter() - ts) * 1e3)
            single_mbs += s.num_mb
        eng1.close(sid)
    single_s = time.perf_counter() - t0
    eng1.destroy()
    single = single_mbs / single_s

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    peak, peak_kind = hbm_peak()
    mean_ms = total_ms / args.steps
    achieved = mb_per_step * ALG_BYTES_PER_MB / (mean_ms * 1e-3) / 1e9
    tr = ncu_traffic_per_mb()
    sad_rate = mb_per_step * SAD_PER_MB / (mean_ms * 1e-3)
    line = {
        "metric": "encoded MB/s (batched 64 mixed QCIF/CIF streams, bit-exact to the reference)",
        "value": value, "unit": "MB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mean_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded pan/object clips, 24-picture ping-pong per stream)",
        "config": {"workload": args.workload, "streams": len(streams), "mb_per_step": mb_per_step,
                   "me_mode": "reference (11x11 grid + 7x7 refinement)",
                   "l2": "flushed before every timed step (256 MiB write)", "parallelism": f"sessions x{world}"},
        "e2e": {"value": e2e, "unit": "MB/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "single_stream": {"value": single, "unit": "MB/s", "pictures": len(single_lat)},
        "batch_vs_single": value / single,
        "latency_ms": {"batched_p50": float(np.percentile(lat, 50)), "batched_p99": float(np.percentile(lat, 99)),
                       "single_p50": float(np.percentile(single_lat, 50)),
                       "single_p99": float(np.percentile(single_lat, 99))},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind,
                     "traffic": (tr * mb_per_step) if tr else None},
        "sad_roofline": {"achieved": sad_rate, "peak": peak_sad, "unit": "absdiff/s", "frac": sad_rate / peak_sad,
                         "peak_source": "project microbenchmark of the search's SAD step"},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        mbs, el = cpu_baseline(streams, 3, threads)
        line["cpu_baseline"] = {"value": mbs / el, "unit": "MB/s", "cores": threads, "kind": "port",
                                "sample": f"{len(streams)} streams x 3 pictures (oracle, C)"}
    print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    if args.impl == "reference":
        reference_arm(args, world, rank)
        if dist:
            dist.destroy_process_group()
        return
    ours(args, world, rank, local, dist)


if __name__ == "__main__":
    main()
