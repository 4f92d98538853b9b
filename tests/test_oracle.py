"""CPU checks of the oracle: its internal consistency, and its agreement with
the reference's own host code (mode decision, bitstream writers) compiled
from the reference sources into oracle/_ref."""
import os
import tempfile

import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import synth


def _zorder_argmin(cost):
    D = cost.shape[0]
    best = None
    for ty in range(D):
        for tx in range(D):
            z = 0
            for b in range(5):
                z |= ((tx >> b) & 1) << (2 * b) | ((ty >> b) & 1) << (2 * b + 1)
            k = (int(cost[ty, tx]), z)
            if best is None or k < best[0]:
                best = (k, tx, ty)
    return best


@pytest.mark.parametrize("D", [7, 11, 31])
def test_tree_equals_zorder_argmin(D):
    """The reference's 2-D tie-break tree (megpu_kernels.cuh:95-154) returns
    the minimum cost and, among ties, the smallest Z-order index; the CUDA
    core relies on this to replace the tree by one warp min-reduction."""
    rng = np.random.default_rng(D)
    for trial in range(300):
        cost = rng.integers(0, 3 + trial % 5, (D, D)).astype(np.uint32)
        cost[rng.random((D, D)) < 0.25] = 65535
        vx = np.tile(np.arange(D, dtype=np.int8), (D, 1))
        vy = vx.T.copy()
        c, x, y = O.tree_reduce(cost, vx, vy)
        (kc, _), tx, ty = _zorder_argmin(cost)
        assert (c, x, y) == (kc, tx, ty)


def test_loop_filter_orders_agree():
    """Setup filters horizontally first, reconstruction vertically first
    (mbgpu_kernels.cuh:84-149 vs :1015-1080); both round identically."""
    rng = np.random.default_rng(3)
    lib = O.lib()
    for _ in range(2000):
        p = rng.integers(0, 256, (10, 12)).astype(np.uint8)
        a = np.zeros(64, np.int32)
        b = np.zeros(64, np.int32)
        lib.orc_loop_filter_hv(O._p(p), 12, 2, 1, O._p(a))
        lib.orc_loop_filter_vh(O._p(p), 12, 2, 1, O._p(b))
        assert np.array_equal(a, b)


def test_dct_of_flat_block():
    for v in (0, 1, 37, 128, 255):
        c = O.fdct(np.full(64, v))
        assert c[0] == 8 * v and not c[1:].any()
        r = O.idct(np.concatenate([[8 * v], np.zeros(63, np.int32)]))
        assert np.all(r == min(255, v))


def test_contraction_touches_only_the_idct():
    """nvcc's default contraction (fmad=1) leaves the forward DCT, hence every
    level and bitstream, unchanged; in the inverse DCT it fuses the left-hand
    prescaled product of the first column-pass adds, which moves a rare
    output by one."""
    rng = np.random.default_rng(11)
    idct_diff = 0
    for _ in range(20000):
        b = rng.integers(-255, 256, 64)
        assert np.array_equal(O.fdct(b, 1), O.fdct(b, 0))
        d = rng.integers(-2048, 2048, 64) * (rng.random(64) < 0.3)
        x, y = O.idct(d, 1), O.idct(d, 0)
        assert np.abs(x - y).max() <= 1
        idct_diff += int(not np.array_equal(x, y))
    assert 0 < idct_diff < 2000


def test_inverse_quant_table():
    for q in range(1, 32):
        assert O.lib().orc_inv_quant(q) == np.float32(1.0 / np.float64(np.float32(2 * q)))


def test_sequence_is_deterministic():
    fr = synth.clip(0, 176, 144, 5, 4)
    a = O.encode_sequence(fr, 176, 144, 8)
    b = O.encode_sequence(fr, 176, 144, 8)
    assert np.array_equal(a["recon"], b["recon"]) and np.array_equal(a["mbs"], b["mbs"])


def test_sequence_psnr_plausible():
    fr = synth.clip(0, 176, 144, 1, 6)
    r = O.encode_sequence(fr, 176, 144, 8)
    fs = 176 * 144
    for i in range(6):
        d = fr[i, :fs].astype(float) - r["recon"][i, :fs]
        psnr = 10 * np.log10(255 ** 2 / (d ** 2).mean())
        assert 30.0 < psnr < 45.0
    # P pictures: most vectors follow the pan (+2, -1)
    mv = r["md"][3]
    assert np.mean((mv["mvx"] == 2) & (mv["mvy"] == -1)) > 0.4


needs_ref = pytest.mark.skipif(not O.have_reference_builds(),
                               reason="oracle/_ref not built (needs the reference sources)")


@needs_ref
@pytest.mark.parametrize("w,h,frames,quant,intra", [(176, 144, 8, 8, 0), (352, 288, 3, 12, 2), (176, 144, 5, 31, 0),
                                                    (176, 144, 5, 1, 3)])
def test_oracle_matches_reference_host_code(w, h, frames, quant, intra):
    """The oracle's sequence loop (its own mode decision) equals the frame
    loop driver that runs the reference's h261_moded.c on the oracle backend,
    and the bitstream written from the oracle's macroblocks by the
    reference's writers equals the driver's bitstream."""
    fr = synth.clip(0, w, h, 2, frames)
    with tempfile.TemporaryDirectory() as td:
        yuv = os.path.join(td, "in.yuv")
        fr.tofile(yuv)
        bits, rec, dump = O.run_driver("oracle", yuv, w, h, frames, td, quant=quant, intra=intra)
        d = O.read_dump(dump)
        recd = np.fromfile(rec, np.uint8).reshape(frames, -1)
        stream = open(bits, "rb").read()
    r = O.encode_sequence(fr, w, h, quant, intra_period=intra)
    assert np.array_equal(recd, r["recon"])
    out = b""
    for i in range(frames):
        assert np.array_equal(d[i]["md"], r["md"][i])
        assert np.array_equal(d[i]["mbs"], r["mbs"][i])
        out += O.write_picture(r["mbs"][i], w, h, i, d[i]["type"], quant)
    assert out == stream


@needs_ref
def test_ratecontrol_stream_runs():
    """CBR through the reference's rate control (config-1 style) on the oracle."""
    fr = synth.clip(1, 352, 288, 4, 6)
    with tempfile.TemporaryDirectory() as td:
        yuv = os.path.join(td, "in.yuv")
        fr.tofile(yuv)
        bits, rec, dump = O.run_driver("oracle", yuv, 352, 288, 6, td, quant=0, bitrate=384000, intra=132)
        d = O.read_dump(dump)
    qs = [f["quant"] for f in d]
    assert all(1 <= q <= 31 for q in qs) and len(set(qs)) >= 1
