"""Edge cases of the search and the coder against the oracle, bit for bit:

* pictures of one to six macroblocks (16x16, 32x16, 16x48, 48x32), where
  every macroblock is a border macroblock and the search limits leave a few
  vectors (one, for a 16x16 picture) -- with the reference search and the
  full search;
* flat content, where every candidate of every search has the same SAD and
  only the reference's tie-break decides the vector;
* saturated content (0 and 255 planes alternating with noise), where the
  prediction, residual and reconstruction clamps are reached.
"""
import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _encode(frames, w, h, quant, me_mode=0, intra=0):
    out_mbs, out_rec = [], []
    with Engine(me_mode=me_mode, warps_per_cta=4, kernel_split=1, tail_items=3, staging=1) as e:
        sid = e.open(w, h, quant, intra_period=intra)
        for i in range(frames.shape[0]):
            e.submit_frame(sid, frames[i])
            e.step()
            e.sync()
            out_mbs.append(e.result(sid).to_abi(w))
            out_rec.append(np.concatenate(e.recon(sid)))
    return out_mbs, out_rec


def _check(frames, w, h, quant, me_mode=0, intra=0, where=""):
    want = O.encode_sequence(frames, w, h, quant, intra_period=intra, me_mode=me_mode)
    got_mbs, got_rec = _encode(frames, w, h, quant, me_mode, intra)
    for i in range(frames.shape[0]):
        g, o = got_mbs[i], want["mbs"][i]
        for f in ("type", "flags", "quant", "cbp", "mv", "tcoeff"):
            assert np.array_equal(g[f], o[f]), f"{where} picture {i}: field {f} differs"
        assert np.array_equal(got_rec[i], want["recon"][i]), f"{where} picture {i}: reconstruction differs"


@pytest.mark.parametrize("w,h", [(16, 16), (32, 16), (16, 48), (48, 32)])
@pytest.mark.parametrize("me_mode", [0, 1])
def test_tiny_pictures(gpu, w, h, me_mode):
    rng = np.random.default_rng(w * 100 + h + me_mode)
    base = rng.integers(0, 256, (h + 32, w + 32), np.uint8)
    frames = []
    for t in range(4):
        # the same texture shifted by a few pixels per picture, plus noise
        y = base[4 + t:4 + t + h, 8 - t:8 - t + w].astype(np.int16)
        y = np.clip(y + rng.integers(-3, 4, y.shape), 0, 255).astype(np.uint8)
        c = rng.integers(0, 256, (2, h // 2, w // 2), np.uint8)
        frames.append(np.concatenate([y.ravel(), c.ravel()]))
    _check(np.stack(frames), w, h, 8, me_mode=me_mode, where=f"{w}x{h} me_mode {me_mode}")


def test_flat_content_all_ties(gpu):
    w, h = 176, 144
    frames = np.full((3, w * h * 3 // 2), 128, np.uint8)
    frames[2, : w * h] = 96   # a flat step in brightness: every vector still ties
    _check(frames, w, h, 8, where="flat")


@pytest.mark.parametrize("quant", [1, 31])
def test_saturated_content(gpu, quant):
    w, h = 176, 144
    rng = np.random.default_rng(quant)
    frames = []
    for t in range(4):
        y = np.where(rng.random((h, w)) < 0.5, 0, 255).astype(np.uint8) if t % 2 else \
            np.where((np.arange(w)[None, :] // 8 + np.arange(h)[:, None] // 8 + t) % 2, 0, 255).astype(np.uint8)
        c = np.where(rng.random((2, h // 2, w // 2)) < 0.5, 0, 255).astype(np.uint8)
        frames.append(np.concatenate([y.ravel(), c.ravel()]))
    _check(np.stack(frames), w, h, quant, intra=3, where=f"saturated QUANT {quant}")
