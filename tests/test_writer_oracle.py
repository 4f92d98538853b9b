"""The oracle's restatement of the reference's bitstream syntax and rate
control (oracle/h261_writer.c), pinned two ways on the CPU:

* against the reference's own writers (src/h261_picture.c, h261_gob.c,
  h261_macroblock.c, compiled unchanged into oracle/_ref/) on random
  macroblock records that reach every MTYPE, MQUANT, escapes, the MVD wrap
  and the MB-address and predictor resets;
* against the golden fixtures (per-picture SHA-256 of the bitstream the
  reference produced on a B200), the rate-controlled case included.
"""
import glob
import json
import os
import sys

import numpy as np
import pytest

import oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)
import make_golden as MG  # noqa: E402

FIXTURES = sorted(glob.glob(os.path.join(HERE, "*.json")))

need_ref = pytest.mark.skipif(not O.have_reference_builds(), reason="reference writers not built (oracle/_ref)")


def random_records(rng, w, h, quant, intra_picture, mq_rate=0.2, esc_rate=0.05):
    """Macroblock records the reference writer accepts."""
    nmb = (w // 16) * (h // 16)
    mbs = np.zeros(nmb, O.MB_DTYPE)
    for i in range(nmb):
        m = mbs[i]
        m["mb_x"], m["mb_y"] = (i % (w // 16)) * 16, (i // (w // 16)) * 16
        m["quant"] = rng.integers(1, 32) if rng.random() < mq_rate else quant
        intra = intra_picture or rng.random() < 0.1
        if intra:
            m["type"], m["flags"], m["cbp"] = 0, 4, 63
        else:
            m["type"] = 2
            m["flags"] = rng.choice([0, 1, 3, 4, 5, 7])
            if m["flags"] & 1:
                m["mv"] = rng.integers(-15, 16, 2)
            if m["flags"] & 4:
                m["cbp"] = rng.integers(1, 64)
        for b in range(6):
            if not intra and not (m["cbp"] & (32 >> b) and m["flags"] & 4):
                continue
            c = np.zeros(64, np.int32)
            nz = rng.integers(0 if intra else 1, 20)
            pos = rng.choice(np.arange(1 if intra else 0, 64), size=nz, replace=False)
            big = rng.random(nz) < esc_rate
            val = np.where(big, rng.integers(16, 128, nz), rng.integers(1, 4, nz))
            c[pos] = val * rng.choice([-1, 1], nz)
            if intra:
                c[0] = rng.integers(1, 256)
            m["tcoeff"][b] = c
    return mbs


@need_ref
@pytest.mark.parametrize("w,h", [(176, 144), (352, 288)])
@pytest.mark.parametrize("seed", range(6))
def test_writer_matches_reference_on_random_records(w, h, seed):
    rng = np.random.default_rng(1000 + seed)
    quant = int(rng.integers(1, 32))
    for frame_num, intra in [(seed * 7, True), (seed * 7 + 1, False), (40 + seed, False)]:
        mbs = random_records(rng, w, h, quant, intra)
        ft = 0 if intra else 1
        want = O.write_picture(mbs, w, h, frame_num, ft, quant)
        got = O.write_picture_oracle(mbs, w, h, frame_num, ft, quant)
        assert got == want, f"picture {frame_num}: {len(got)} vs {len(want)} bytes"


@need_ref
def test_writer_matches_reference_on_edge_records():
    """Uncoded GOBs, runs of skipped MBs of every length, vectors whose
    difference wraps, first inter coefficients of +-1 and larger."""
    rng = np.random.default_rng(7)
    w, h, q = 352, 288, 9
    mbs = np.zeros(396, O.MB_DTYPE)
    mbs["type"] = 2
    mbs["quant"] = q
    # GOB 1 (MB rows 0-2, left half) stays empty; elsewhere every 3rd MB is coded
    for i in range(396):
        gx, gy = (i % 22) // 11, (i // 22) // 3
        if gy == 0 and gx == 0:
            continue
        if i % 3 == 0 or i % 7 == 0:
            m = mbs[i]
            m["flags"] = 5
            m["mv"] = (15, -15) if i % 2 else (-15, 15)
            m["cbp"] = 32
            m["tcoeff"][0][0] = [1, -1, 2, -3, 127, -127][i % 6]
            m["tcoeff"][0][63] = 1
    for fnum in (0, 31, 32):
        assert O.write_picture_oracle(mbs, w, h, fnum, 1, q) == O.write_picture(mbs, w, h, fnum, 1, q)


def test_writer_refuses_what_the_reference_cannot_write():
    mbs = np.zeros(99, O.MB_DTYPE)
    mbs["type"], mbs["quant"] = 2, 8
    mbs[5]["flags"], mbs[5]["cbp"] = 4, 0            # COEFF without a coded block
    with pytest.raises(ValueError):
        O.write_picture_oracle(mbs, 176, 144, 0, 1, 8)
    mbs[5]["cbp"] = 32                                # a coded block of zeros
    with pytest.raises(ValueError):
        O.write_picture_oracle(mbs, 176, 144, 0, 1, 8)
    with pytest.raises(ValueError):
        O.write_picture_oracle(np.zeros(80, O.MB_DTYPE), 160, 128, 0, 1, 8)


def test_zigzag_is_a_permutation_in_diagonal_order():
    z = O.zigzag()
    assert sorted(z.tolist()) == list(range(64))
    diag = [(p // 8) + (p % 8) for p in z]
    assert diag == sorted(diag)


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-5] for p in FIXTURES])
def test_stream_matches_reference_fixture(path):
    """The oracle's whole frame loop (core + writer + rate control) yields the
    reference's bitstream, picture by picture."""
    g = json.load(open(path))
    opt = g["options"]
    fr = MG.make_input(g["case"])
    assert MG.sha(fr.tobytes()) == g["input_sha256"]
    bits, nb, nq, recon = O.encode_stream(fr, g["width"], g["height"], quant=opt.get("quant", 0),
                                          bitrate=opt.get("bitrate", 384000), intra_period=opt.get("intra", 0))
    off = 0
    for i, want in enumerate(g["per_frame"]):
        assert nq[i] == want["quant"], f"picture {i}: QUANT {nq[i]} != {want['quant']}"
        assert nb[i] == want["bytes"], f"picture {i}: {nb[i]} != {want['bytes']} bytes"
        assert MG.sha(bits[off:off + nb[i]]) == want["bits"], f"picture {i}: bitstream"
        assert MG.sha(recon[i].tobytes()) == want["recon"], f"picture {i}: reconstruction"
        off += nb[i]
    assert MG.sha(bits) == g["stream_sha256"]


def test_rate_control_reacts_to_size():
    """Pictures far over budget raise QUANT; far under budget lower it."""
    rc = O.RateControl(10, 384000)
    q0 = rc.picture_quant(1, 396 * 300, 396)
    for _ in range(4):
        rc.update(1, q0, 60000)
    q_big = rc.picture_quant(1, 396 * 300, 396)
    rc2 = O.RateControl(10, 384000)
    q1 = rc2.picture_quant(1, 396 * 300, 396)
    for _ in range(4):
        rc2.update(1, q1, 200)
    q_small = rc2.picture_quant(1, 396 * 300, 396)
    assert q_big > q_small and 1 <= q_small <= 31 and 1 <= q_big <= 31
