"""The device bitstream writer: every picture's H.261 bytes must be the
reference's.  Pinned against the golden fixtures (per-picture SHA-256 of the
bitstream the reference produced on a B200) and against the oracle's
restatement of the reference writers on the engine's own records."""
import ctypes
import glob
import json
import os
import sys

import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import synth
from h261enc_cuda_b200.engine import Engine

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)
import make_golden as MG  # noqa: E402

pytestmark = pytest.mark.gpu
FIXTURES = sorted(glob.glob(os.path.join(HERE, "*.json")))
IDS = [os.path.basename(p)[:-5] for p in FIXTURES]


@pytest.mark.parametrize("levels_to_host", [1, 0])
@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_bitstream_matches_reference_fixture(gpu, path, levels_to_host):
    """Fixed-QUANT cases as they are; the rate-controlled case with the
    QUANT sequence the reference's rate control chose."""
    g = json.load(open(path))
    opt = g["options"]
    fr = MG.make_input(g["case"])
    w, h = g["width"], g["height"]
    with Engine(warps_per_cta=4, levels_to_host=levels_to_host) as e:
        sid = e.open(w, h, max(opt.get("quant", 0), 1), intra_period=opt.get("intra", 0), bitstream=1)
        stream = b""
        for i, want in enumerate(g["per_frame"]):
            e.submit_frame(sid, fr[i], quant=want["quant"])
            e.step()
            e.sync()
            r = e.result(sid)
            assert r.bits_status == 0
            assert (r.levels is None) == (levels_to_host == 0)
            assert len(r.bits) == want["bytes"], f"picture {i}: {len(r.bits)} != {want['bytes']} bytes"
            assert MG.sha(r.bits) == want["bits"], f"picture {i}: bitstream differs"
            stream += r.bits
    assert MG.sha(stream) == g["stream_sha256"]


@pytest.mark.parametrize("preset,w,h,quant", [(0, 176, 144, 1), (1, 352, 288, 2), (3, 176, 144, 5),
                                              (2, 352, 288, 17), (0, 176, 144, 31)])
def test_bitstream_matches_oracle_writer(gpu, preset, w, h, quant):
    fr = synth.clip(preset, w, h, 50 + quant, 5)
    with Engine(warps_per_cta=4) as e:
        sid = e.open(w, h, quant, intra_period=3, bitstream=1)
        for i in range(fr.shape[0]):
            e.submit_frame(sid, fr[i])
            e.step()
            e.sync()
            r = e.result(sid)
            want = O.write_picture_oracle(r.to_abi(w), w, h, i, r.frame_type, quant)
            assert r.bits == want, f"picture {i}: {len(r.bits)} vs {len(want)} bytes"
            # the per-MB coefficient counts add up to the picture
            assert int(r.mbs["coef_bits"].sum()) < 8 * len(r.bits)


def test_bitstream_batch_pipelined_matches_oracle_stream(gpu):
    """Mixed sessions, steps issued back to back, results read one step late."""
    specs = [(176, 144, 8, 31), (352, 288, 12, 32), (176, 144, 3, 33), (352, 288, 24, 34), (176, 144, 16, 35)]
    n = 6
    clips = [synth.clip(2, w, h, seed, n) for (w, h, q, seed) in specs]
    want = [O.encode_stream(c, w, h, quant=q)[0] for c, (w, h, q, _) in zip(clips, specs)]
    got = [b"" for _ in specs]
    with Engine(warps_per_cta=4, levels_to_host=0) as e:
        sids = [e.open(w, h, q, bitstream=1) for (w, h, q, _) in specs]
        for i in range(n + 1):
            if i < n:
                e.submit_frames(sids, [c[i] for c in clips])
                e.step()
            if i > 0:
                e.wait_previous() if i < n else e.sync()
                total = 0
                for k, sid in enumerate(sids):
                    r = e.result(sid)
                    assert r.frame_index == i - 1
                    got[k] += r.bits
                    total += len(r.bits)
                assert e.step_bits() == (total, len(sids))
    for k in range(len(specs)):
        assert got[k] == want[k], f"session {k}"


def test_bitstream_host_arena_overflow_falls_back(gpu):
    """A host arena too small for a step: the pictures that miss it are read
    from the device slots, later steps get a larger arena."""
    fr = synth.clip(1, 352, 288, 7, 4)
    want = O.encode_stream(fr, 352, 288, quant=2)[1]
    with Engine(warps_per_cta=4, bits_host_bytes=4096) as e:
        a = e.open(352, 288, 2, bitstream=1)
        b = e.open(352, 288, 2, bitstream=1)
        for i in range(fr.shape[0]):
            e.submit_frames([a, b], [fr[i], fr[i]])
            e.step()
            e.sync()
            ra, rb = e.result(a), e.result(b)
            assert len(ra.bits) == want[i] and ra.bits == rb.bits


def test_bitstream_refused_for_other_sizes(gpu):
    with Engine(warps_per_cta=4) as e:
        with pytest.raises(RuntimeError):
            e.open(320, 240, 8, bitstream=1)
        sid = e.open(320, 240, 8)          # the core itself takes any multiple of 16
        e.submit_frame(sid, synth.clip(0, 320, 240, 1, 1)[0])
        e.step()
        e.sync()
        assert e.result(sid).bits is None


def test_rate_control_on_device_matches_reference_fixture(gpu):
    """The rate-controlled golden case with the rate control on the device:
    QUANT per picture, bytes and bitstream as the reference chose them."""
    path = os.path.join(HERE, "cif_scenes_cbr384k.json")
    g = json.load(open(path))
    opt = g["options"]
    fr = MG.make_input(g["case"])
    w, h = g["width"], g["height"]
    with Engine(warps_per_cta=4, levels_to_host=0) as e:
        sid = e.open(w, h, 10, intra_period=opt["intra"], bitstream=1, rate_control=1, bitrate=opt["bitrate"])
        for i, want in enumerate(g["per_frame"]):
            e.submit_frame(sid, fr[i])
            e.step()
            e.sync()
            r = e.result(sid)
            assert r.quant == want["quant"], f"picture {i}: QUANT {r.quant} != {want['quant']}"
            assert MG.sha(r.bits) == want["bits"], f"picture {i}: bitstream differs"


def test_rate_control_mixed_batch_pipelined_matches_oracle(gpu):
    """CBR and fixed-QUANT sessions in the same steps, issued back to back:
    every stream equals the oracle's frame loop with its own settings."""
    specs = [(352, 288, 0, 256000, 41), (176, 144, 9, 0, 42), (176, 144, 0, 64000, 43), (352, 288, 14, 0, 44),
             (352, 288, 0, 512000, 45)]
    n = 8
    clips = [synth.clip(1 if w == 352 else 2, w, h, seed, n) for (w, h, q, b, seed) in specs]
    want = [O.encode_stream(c, w, h, quant=q, bitrate=b or 384000, intra_period=5)
            for c, (w, h, q, b, _) in zip(clips, specs)]
    got = [b"" for _ in specs]
    quants = [[] for _ in specs]
    with Engine(warps_per_cta=4, levels_to_host=0) as e:
        sids = [e.open(w, h, q or 10, intra_period=5, bitstream=1, rate_control=1 if b else 0, bitrate=b)
                for (w, h, q, b, _) in specs]
        for i in range(n + 1):
            if i < n:
                e.submit_frames(sids, [c[i] for c in clips])
                e.step()
            if i > 0:
                e.wait_previous() if i < n else e.sync()
                for k, sid in enumerate(sids):
                    r = e.result(sid)
                    got[k] += r.bits
                    quants[k].append(r.quant)
    for k in range(len(specs)):
        assert quants[k] == list(want[k][2]), f"session {k}: QUANTs {quants[k]} vs {list(want[k][2])}"
        assert got[k] == want[k][0], f"session {k}: bitstream"


def test_rate_control_skipping_steps_two_behind_matches_oracle(gpu):
    """CBR sessions that skip steps, with three steps in flight and the host
    reading two behind: a session's rate control reads the size of its
    previous picture, which may be two steps back on another stream, and
    every stream still equals the oracle's frame loop."""
    specs = [(352, 288, 256000, 51, 1), (176, 144, 64000, 52, 2), (176, 144, 96000, 53, 3)]
    steps = 12
    clips = [synth.clip(1 if w == 352 else 2, w, h, seed, steps) for (w, h, b, seed, every) in specs]
    got = [b"" for _ in specs]
    used = [0 for _ in specs]
    with Engine(warps_per_cta=4, levels_to_host=0) as e:
        sids = [e.open(w, h, 10, bitstream=1, rate_control=1, bitrate=b) for (w, h, b, _, _) in specs]

        def read(k):
            e.wait_step(k)
            pics, _ = e.step_pictures(8)
            for p in pics:
                j = sids.index(int(p["session_id"]))
                assert p["status"] in (0, 1)
                got[j] += (ctypes.string_at(int(p["bits"]), int(p["bytes"])) if p["status"] == 0
                           else e.result(int(p["session_id"]), copy=False).bits)

        for k in range(steps):
            live = [j for j, spec in enumerate(specs) if k % spec[4] == 0]
            e.submit_frames([sids[j] for j in live], [clips[j][used[j]] for j in live])
            for j in live:
                used[j] += 1
            e.step()
            if k >= 2:
                read(k - 2)
        read(steps - 2)
        read(steps - 1)
    for j, (w, h, b, _, _) in enumerate(specs):
        want = O.encode_stream(clips[j][:used[j]], w, h, quant=0, bitrate=b)[0]
        assert got[j] == want, f"session {j}: bitstream"


def test_rate_control_needs_bitstream(gpu):
    with Engine(warps_per_cta=4) as e:
        with pytest.raises(RuntimeError):
            e.open(176, 144, 10, rate_control=1, bitrate=64000)
        with pytest.raises(RuntimeError):
            e.open(176, 144, 10, bitstream=1, rate_control=1, bitrate=0)


@pytest.mark.parametrize("preset,w,h,quant,bitrate", [(0, 176, 144, 8, 0), (1, 352, 288, 10, 384000),
                                                      (3, 176, 144, 2, 0), (2, 352, 288, 20, 0)])
def test_decoded_bitstream_is_the_device_reconstruction(gpu, preset, w, h, quant, bitrate):
    """The conformance decoder turns the device's bitstream back into the
    device's own reconstructions, picture by picture."""
    fr = synth.clip(preset, w, h, 60 + quant, 7)
    stream, recs = b"", []
    with Engine(warps_per_cta=4, levels_to_host=0) as e:
        sid = e.open(w, h, quant, intra_period=4, bitstream=1, rate_control=1 if bitrate else 0, bitrate=bitrate)
        for i in range(fr.shape[0]):
            e.submit_frame(sid, fr[i])
            e.step()
            e.sync()
            stream += e.result(sid).bits
            recs.append(np.concatenate(e.recon(sid)))
    drec, dmbs, dw, dh = O.decode_stream(stream)
    assert (dw, dh) == (w, h) and drec.shape[0] == len(recs)
    for i in range(len(recs)):
        assert np.array_equal(drec[i], recs[i]), f"picture {i}: decoded picture differs"
