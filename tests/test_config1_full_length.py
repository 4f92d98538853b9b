"""The plain single-stream CIF configuration at its full length: 352x288,
300 pictures, an intra picture every 132 (pictures 0 and 132, and 264), CBR
rate control at 384 kbit/s, content whose pan is redrawn every 30 pictures
with a scene cut (new seed) at picture 150.  At 384 kbit/s this content
drives the rate control to QUANT 31 for most pictures; the 2 Mbit/s variant
keeps QUANT moving (13..26) through the intra refresh and the scene cut, so
the rate control's per-type prediction state (h261_ratectrl.c:144-222) is
exercised in both regimes.

* CPU: the oracle's frame loop (its restatement of the rate control and the
  writers) equals the reference's own host code -- h261_ratectrl.c,
  h261_moded.c and the writers, compiled unchanged -- driven over the CPU
  oracle, picture by picture (bytes, QUANT, reconstructions, boundary dumps).
* GPU: the batched engine (device rate control and bitstream writer) and the
  drop-in boundary (libh261b.so under the reference's host code) equal the
  oracle, and the reference's own CUDA built for sm_100a equals both, over all
  300 pictures.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import synth
from h261enc_cuda_b200.engine import Engine

W, H, N, INTRA, SEED = 352, 288, 300, 132, 2026
CASES = [384000, 2000000]

_clip = None
_want = {}


def clip():
    global _clip
    if _clip is None:
        _clip = synth.clip(synth.PRESET_CIF_SCENES, W, H, SEED, N)
    return _clip


def oracle_stream(bitrate):
    if bitrate not in _want:
        _want[bitrate] = O.encode_stream(clip(), W, H, quant=0, bitrate=bitrate, intra_period=INTRA)
    return _want[bitrate]


def split_pictures(bits, nb):
    out, off = [], 0
    for n in nb:
        out.append(bits[off:off + int(n)])
        off += int(n)
    return out


needs_drivers = pytest.mark.skipif(not os.path.exists(O.DRIVERS["oracle"]),
                                   reason="the reference's host code is not built (oracle/_ref)")


def _run(kind, bitrate, td, env=None):
    yuv = os.path.join(td, "in.yuv")
    if not os.path.exists(yuv):
        clip().tofile(yuv)
    b, rc, d = O.run_driver(kind, yuv, W, H, N, td, bitrate=bitrate, intra=INTRA, env=env)
    return open(b, "rb").read(), np.fromfile(rc, np.uint8).reshape(N, -1), O.read_dump(d)


@needs_drivers
@pytest.mark.parametrize("bitrate", CASES)
def test_oracle_frame_loop_equals_reference_host_code(bitrate):
    bits, nb, nq, rec = oracle_stream(bitrate)
    with tempfile.TemporaryDirectory() as td:
        rbits, rrec, dump = _run("oracle", bitrate, td)
    assert len(dump) == N
    assert [d["quant"] for d in dump] == nq.tolist(), "picture QUANT differs from the reference's rate control"
    assert [d["bytes"] for d in dump] == nb.tolist(), "picture sizes differ"
    assert rbits == bits, "bitstreams differ"
    assert np.array_equal(rrec, rec), "reconstructions differ"
    # the configuration reaches what it is meant to: intra pictures at 0,
    # 132 and 264 under rate control
    assert sum(d["type"] == 0 for d in dump) == 3


@pytest.mark.gpu
@pytest.mark.parametrize("bitrate", CASES)
def test_engine_full_length_equals_oracle(gpu, bitrate):
    """300 steps of one CBR session through the batched engine: every
    picture's bytes, QUANT and reconstruction."""
    bits, nb, nq, rec = oracle_stream(bitrate)
    want = split_pictures(bits, nb)
    fr = clip()
    with Engine(max_sessions=4) as e:
        sid = e.open(W, H, 10, intra_period=INTRA, bitstream=1, rate_control=1, bitrate=bitrate)
        for i in range(N):
            e.submit_frame(sid, fr[i])
            e.step()
            e.sync()
            r = e.result(sid)
            assert r.bits_status == 0, f"picture {i}: bitstream status {r.bits_status}"
            assert r.quant == nq[i], f"picture {i}: QUANT {r.quant}, the oracle's rate control chose {nq[i]}"
            assert r.bits == want[i], f"picture {i}: bytes differ"
            assert np.array_equal(np.concatenate(e.recon(sid)), rec[i]), f"picture {i}: reconstruction differs"


needs_ref_cuda = pytest.mark.skipif(
    not all(os.path.exists(O.DRIVERS[k]) for k in ("refgpu", "ours", "oracle")),
    reason="the reference CUDA drivers are not built")


@pytest.mark.gpu
@needs_ref_cuda
@pytest.mark.parametrize("bitrate", CASES)
def test_drop_in_and_reference_cuda_full_length(gpu, bitrate):
    """The reference's frame loop and host code over three device paths --
    the reference's own CUDA (sm_100a), this core behind gpu_device.h, the
    CPU oracle -- write the same 300 pictures: bytes, reconstructions and
    every boundary value (vectors, costs, mode decisions, levels, QUANT)."""
    with tempfile.TemporaryDirectory() as td:
        ob, orec, od = _run("oracle", bitrate, td)
        rb, rrec, rd = _run("refgpu", bitrate, td)
        gb, grec, gd = _run("ours", bitrate, td)
    assert len(rd) == len(gd) == len(od) == N
    assert gb == rb == ob, "bitstreams differ"
    assert np.array_equal(grec, rrec) and np.array_equal(grec, orec), "reconstructions differ"
    for i, (g, r) in enumerate(zip(gd, rd)):
        assert g["quant"] == r["quant"] and g["bytes"] == r["bytes"], f"picture {i}"
        assert np.array_equal(g["me"], r["me"]), f"picture {i}: ME results differ"
        assert np.array_equal(g["md"], r["md"]), f"picture {i}: mode decisions differ"
        assert np.array_equal(g["mbs"], r["mbs"]), f"picture {i}: macroblocks differ"
