"""Parity at the benchmark's full sizes, through properties that do not need
the oracle to encode every stream: every stream's device bitstream, decoded
by the conformance decoder, is the device's own reconstruction picture by
picture, and a sample of the streams equals the oracle's frame loop.

* batch64: the 64 mixed QCIF/CIF streams of the bench in one step each;
* stress1024: the 1024 QCIF streams of the motion-search stress workload.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import workloads
from h261enc_cuda_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _encode_all(streams, pictures, sample):
    clips = [workloads.make_clip(s, pictures) for s in streams]
    bits = [b"" for _ in streams]
    recs = [[] for _ in streams]
    with Engine(max_sessions=len(streams), levels_to_host=0) as e:
        sids = [e.open(s.width, s.height, s.quant, bitstream=1) for s in streams]
        for i in range(pictures):
            e.submit_frames(sids, [c[i] for c in clips])
            assert e.step() == len(streams)
            e.sync()
            pics, span = e.step_pictures(len(streams) + 8)
            assert pics.size == len(streams)
            by_sid = {int(p["session_id"]): p for p in pics}
            for k, sid in enumerate(sids):
                p = by_sid[sid]
                if p["status"] == 0:
                    bits[k] += ctypes.string_at(int(p["bits"]), int(p["bytes"]))
                else:
                    assert p["status"] == 1
                    bits[k] += e.result(sid, copy=False).bits
                recs[k].append(np.concatenate(e.recon(sid)))
    # every stream: its bitstream decodes to its reconstructions
    for k, s in enumerate(streams):
        dec, _, w, h = O.decode_stream(bits[k])
        assert (w, h) == (s.width, s.height) and dec.shape[0] == pictures, f"stream {k}"
        for i in range(pictures):
            assert np.array_equal(dec[i], recs[k][i]), f"stream {k} picture {i}: decode != reconstruction"
    # a sample: the oracle's frame loop on the same pictures
    for k in sample:
        s = streams[k]
        want = O.encode_stream(clips[k], s.width, s.height, quant=s.quant)[0]
        assert bits[k] == want, f"stream {k}: bitstream differs from the oracle"


def test_batch64_full_step_round_trips(gpu):
    streams = workloads.batch64()
    _encode_all(streams, 3, sample=[0, 17, 39, 40, 52, 63])


def test_stress1024_full_step_round_trips(gpu):
    streams = workloads.stress1024()
    _encode_all(streams, 2, sample=[0, 255, 511, 1023])
