"""TEST INFRASTRUCTURE: the reference's own CUDA (oracle/_ref/h261_drive_refgpu,
src/gpu_device.cu built for sm_100a) and this project's core behind the same
gpu_device.h boundary (oracle/_ref/h261_drive_ours), timed picture by picture
on the same seeded clips by the one frame-loop driver (oracle/ref_driver.c,
timing=).  Both write the same bitstream; the script checks that, then
prints per-picture times and MB/s (the first picture, which creates the CUDA
context, is left out).

    python oracle/time_drivers.py [frames]

Needs a GPU and the drivers built by `make -C oracle ref ours`.
"""
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402
from h261enc_cuda_b200 import synth  # noqa: E402

CASES = [
    # name, preset, width, height, quant (0: CBR 384 kbit/s), seed
    ("qcif_q8", synth.PRESET_PAN, 176, 144, 8, 2026),
    ("cif_cbr384", synth.PRESET_CIF_SCENES, 352, 288, 0, 2027),
]


def time_driver(kind: str, preset: int, w: int, h: int, q: int, seed: int, frames: int, tmp: str):
    """Encode one seeded clip with one driver, timing every picture: per
    picture ms (the first left out), MB/s and the bitstream's SHA-256."""
    clip = synth.clip(preset, w, h, seed, frames)
    d = os.path.join(tmp, f"{kind}_{w}x{h}_{q}_{seed}_{frames}")
    os.makedirs(d, exist_ok=True)
    yuv = os.path.join(d, "in.yuv")
    clip.tofile(yuv)
    timing = os.path.join(d, "timing.txt")
    bits = os.path.join(d, "out.h261")
    args = [O.DRIVERS[kind], f"in={yuv}", f"w={w}", f"h={h}", f"frames={frames}", f"bits={bits}",
            f"recon={os.path.join(d, 'recon.yuv')}", f"dump={os.path.join(d, 'dump.bin')}",
            f"timing={timing}", "intra=132" if q == 0 else "intra=0",
            f"quant={q}" if q > 0 else "bitrate=384000"]
    subprocess.run(args, check=True, stdout=subprocess.DEVNULL, timeout=600)
    ms = [float(x) for x in open(timing).read().split()]
    steady = ms[1:]
    nmb = (w // 16) * (h // 16)
    return {"ms_per_picture_median": statistics.median(steady), "ms_per_picture_mean": statistics.mean(steady),
            "ms_per_picture_p99": sorted(steady)[min(len(steady) - 1, int(0.99 * len(steady)))],
            "mb_per_s": nmb * len(steady) / (sum(steady) * 1e-3), "pictures": len(steady),
            "sha256": hashlib.sha256(open(bits, "rb").read()).hexdigest()}


def run(frames: int):
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, preset, w, h, q, seed in CASES:
            row = {kind: time_driver(kind, preset, w, h, q, seed, frames, tmp) for kind in ("refgpu", "ours")}
            row["same_bitstream"] = row["refgpu"].pop("sha256") == row["ours"].pop("sha256")
            row["speedup"] = row["ours"]["mb_per_s"] / row["refgpu"]["mb_per_s"]
            out[name] = row
    return out


if __name__ == "__main__":
    frames = int(sys.argv[1]) if len(sys.argv) > 1 else 30
    print(json.dumps(run(frames), indent=1))
