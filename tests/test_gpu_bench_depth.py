"""Parity at the depth the benchmark runs, every stream against the oracle.

The bench's own stream bookkeeping (bench.Runner: each stream plays a seeded
clip forwards and backwards, a stream that reaches its length is replaced by
a new session that starts with an intra picture, and the old one is closed
only once its last step has been read) drives the engine with three steps in
flight, reading step k-2 after issuing step k, pictures queued alternately
from HBM and from host memory (the value and the end-to-end paths), steps
replayed from CUDA graphs once their launch signature repeats.  Every
picture of every session -- bitstream bytes, in order -- and every session's
final reconstruction must equal the oracle's frame loop on the same
pictures.

* batch64: all 64 mixed QCIF/CIF streams for 64 steps (a ping-pong reversal
  at picture 24, and the streams shorter than 64 pictures restart);
* stress1024: all 1024 QCIF random-motion streams for 4 steps.
"""
import ctypes
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import bench
import oracle as O
from h261enc_cuda_b200 import workloads
from h261enc_cuda_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _run_pipelined(streams, steps, clip_len):
    """Every picture's bytes per session instance (slot, generation), the
    pictures each instance received, and each live instance's final
    reconstruction."""
    pools = bench.device_clips(streams, clip_len, 0)
    eng = Engine(device=0, max_sessions=4 * len(streams), levels_to_host=0)
    try:
        sizes = {}
        for s in streams:
            sizes[(s.width, s.height)] = sizes.get((s.width, s.height), 0) + 1
        for (w, h), k in sizes.items():
            eng.reserve(w, h, 2 * k, bitstream=1)
        run = bench.Runner(eng, streams, pools, clip_len=clip_len)
        gen = np.zeros(len(streams), np.int64)
        owner = []                # per step: session id -> (slot, generation)
        got = {}                  # (slot, generation) -> [bytes of picture 0, 1, ...]
        first = run.queued

        def consume(k):
            eng.wait_step(first + k)
            pics, _ = eng.step_pictures(len(streams) + 8)
            assert pics.size == len(streams), f"step {k}: {pics.size} pictures"
            for p in pics:
                sid = int(p["session_id"])
                key = owner[k][sid]
                if p["status"] == 0:
                    b = ctypes.string_at(int(p["bits"]), int(p["bytes"]))
                else:
                    assert p["status"] == 1, f"step {k} session {sid}: status {p['status']}"
                    b = eng.result(sid, copy=False).bits
                lst = got.setdefault(key, [])
                assert int(p["frame_index"]) == len(lst), f"step {k} {key}: picture out of order"
                lst.append(b)
            run.retire(first + k)

        for it in range(steps):
            before = run.sids.copy()
            # alternate in blocks of 12 steps: each of the engine's three
            # step slots then meets the same launch signature four times in
            # a row (launched, captured, replayed twice)
            if (it // 12) % 2:
                run.queue_host(wait=False)
            else:
                run.queue_device()
            gen += run.sids != before
            owner.append({int(run.sids[j]): (j, int(gen[j])) for j in range(len(streams))})
            assert eng.step() == len(streams)
            if it >= 2:
                consume(it - 2)
        for k in range(max(0, steps - 2), steps):
            consume(k)
        eng.sync()
        final = {}
        for j in range(len(streams)):
            y, cb, cr = eng.recon(int(run.sids[j]))
            final[(j, int(gen[j]))] = np.concatenate([y, cb, cr])
        captures, replays = eng.graph_stats()
    finally:
        eng.destroy()
    return got, final, [p[1] for p in pools], (captures, replays)


def _check_against_oracle(streams, got, final, clips, clip_len):
    index = [workloads.clip_index(k, clip_len) for k in range(10000)]

    def one(item):
        (slot, g), pics = item
        s = streams[slot]
        frames = clips[slot][index[:len(pics)]]
        bits, nb, _, rec = O.encode_stream(frames, s.width, s.height, quant=s.quant)
        off, bad = 0, []
        for i, n in enumerate(nb):
            if pics[i] != bits[off:off + int(n)]:
                bad.append(i)
            off += int(n)
        rec_ok = (slot, g) not in final or np.array_equal(final[(slot, g)], rec[-1])
        return (slot, g), bad, rec_ok

    O.lib()
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        results = list(ex.map(one, sorted(got.items())))
    for key, bad, rec_ok in results:
        assert not bad, f"stream {key}: pictures {bad[:8]} differ from the oracle"
        assert rec_ok, f"stream {key}: final reconstruction differs from the oracle"
    return len(results)


def test_batch64_every_stream_at_bench_depth(gpu):
    streams = workloads.batch64()
    steps = 64
    got, final, clips, (captures, replays) = _run_pipelined(streams, steps, bench.CLIP_LEN)
    assert sum(len(v) for v in got.values()) == steps * len(streams)
    restarted = [k for k in got if k[1] > 0]
    assert restarted, "no stream restarted within the run"
    assert replays > 0, "no step replayed a CUDA graph"
    n = _check_against_oracle(streams, got, final, clips, bench.CLIP_LEN)
    assert n == len(streams) + len(restarted)


def test_stress1024_every_stream(gpu):
    streams = workloads.stress1024()
    steps = 4
    got, final, clips, _ = _run_pipelined(streams, steps, steps)
    assert len(got) == len(streams) and all(len(v) == steps for v in got.values())
    _check_against_oracle(streams, got, final, clips, steps)
