"""Make the golden fixtures of this directory from the reference itself.

The reference project ships no test vectors, so the fixtures are outputs of
its own code: src/gpu_device.cu and its host sources, compiled unchanged for
sm_100a by oracle/Makefile (oracle/_ref/h261_drive_refgpu, the frame-loop
driver on the reference's CUDA), run on a B200 over the seeded cases below.
For every picture a fixture records the SHA-256 of the bitstream bytes, of
the reconstruction and of the boundary records (motion estimation results,
mode decisions, macroblocks with their levels), plus the SHA-256 of the
generated input, so a test can regenerate the input and compare.

usage (on a GPU box): python tests/golden/make_golden.py OUT_DIR [--driver refgpu]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# name: (source, width, height, seed, frames, driver options)
#   source: ("synth", preset) or ("noise",) -- uniform random bytes
CASES = {
    "qcif_pan_q8": (("synth", 0), 176, 144, 1, 30, {"quant": 8}),
    "cif_scenes_cbr384k": (("synth", 1), 352, 288, 3, 20, {"quant": 0, "bitrate": 384000, "intra": 132}),
    "cif_noise_intra_q1": (("noise",), 352, 288, 5, 10, {"quant": 1, "intra": 1}),
    "cif_noise_intra_q3": (("noise",), 352, 288, 5, 10, {"quant": 3, "intra": 1}),
    "qcif_blockmotion_q12": (("synth", 3), 176, 144, 4, 12, {"quant": 12}),
    "qcif_pan_q1": (("synth", 0), 176, 144, 2, 6, {"quant": 1}),
    "qcif_pan_q31": (("synth", 0), 176, 144, 2, 6, {"quant": 31}),
}


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()


def make_input(case: str) -> np.ndarray:
    (src, w, h, seed, n, _) = CASES[case]
    if src[0] == "noise":
        rng = np.random.default_rng(seed)
        return rng.integers(0, 256, (n, w * h * 3 // 2), dtype=np.uint8)
    from h261enc_cuda_b200 import synth
    return synth.clip(src[1], w, h, seed, n)


def per_frame_record(frames, bits: bytes, recon: np.ndarray):
    out, off = [], 0
    for i, f in enumerate(frames):
        nb = f["bytes"]
        out.append({
            "type": f["type"], "quant": f["quant"], "bytes": nb,
            "bits": sha(bits[off:off + nb]),
            "recon": sha(recon[i].tobytes()),
            "me": sha(f["me"].tobytes()), "md": sha(f["md"].tobytes()), "mbs": sha(f["mbs"].tobytes()),
        })
        off += nb
    assert off == len(bits)
    return out


def run_case(case: str, driver: str, env=None):
    import oracle as O
    (src, w, h, seed, n, opts) = CASES[case]
    fr = make_input(case)
    with tempfile.TemporaryDirectory() as td:
        yuv = os.path.join(td, "in.yuv")
        fr.tofile(yuv)
        bits, rec, dump = O.run_driver(driver, yuv, w, h, n, td, env=env, **opts)
        frames = O.read_dump(dump)
        recon = np.fromfile(rec, np.uint8).reshape(n, -1)
        stream = open(bits, "rb").read()
    return {"case": case, "width": w, "height": h, "frames": n, "options": opts,
            "source": list(src), "seed": seed, "input_sha256": sha(fr.tobytes()),
            "stream_sha256": sha(stream), "per_frame": per_frame_record(frames, stream, recon)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out_dir")
    ap.add_argument("--driver", default="refgpu")
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    a = ap.parse_args()
    os.makedirs(a.out_dir, exist_ok=True)
    for c in a.cases:
        rec = run_case(c, a.driver)
        rec["made_with"] = f"oracle/_ref/h261_drive_{a.driver}"
        with open(os.path.join(a.out_dir, c + ".json"), "w") as f:
            json.dump(rec, f, indent=1)
        print(c, rec["stream_sha256"][:16], len(rec["per_frame"]))


if __name__ == "__main__":
    main()
