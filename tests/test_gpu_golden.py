"""The sm_100a core against the reference itself: the golden fixtures hold
per-picture SHA-256s of the reference's own CUDA build run on a B200
(tests/golden/make_golden.py).  Fixed-QUANT cases go through the batched
engine; every case also goes through the reference's unchanged host code
linked against libh261b.so (the drop-in path)."""
import glob
import json
import os
import sys

import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200.engine import Engine

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)
import make_golden as MG  # noqa: E402

pytestmark = pytest.mark.gpu
FIXTURES = sorted(glob.glob(os.path.join(HERE, "*.json")))
IDS = [os.path.basename(p)[:-5] for p in FIXTURES]


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_engine_matches_reference_fixture(gpu, path):
    g = json.load(open(path))
    opt = g["options"]
    if opt.get("quant", 0) <= 0:
        pytest.skip("rate-controlled case: covered through the drop-in driver")
    fr = MG.make_input(g["case"])
    assert MG.sha(fr.tobytes()) == g["input_sha256"]
    w, h = g["width"], g["height"]
    with Engine(warps_per_cta=4) as e:
        sid = e.open(w, h, opt["quant"], intra_period=opt.get("intra", 0))
        for i, want in enumerate(g["per_frame"]):
            e.submit_frame(sid, fr[i])
            e.step()
            e.sync()
            mbs = e.result(sid).to_abi(w)
            rec = np.concatenate(e.recon(sid))
            assert MG.sha(mbs.tobytes()) == want["mbs"], f"picture {i}: macroblock records"
            assert MG.sha(rec.tobytes()) == want["recon"], f"picture {i}: reconstruction"


@pytest.mark.skipif(not os.path.exists(O.DRIVERS["ours"]), reason="drop-in driver not built")
@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_dropin_driver_matches_reference_fixture(gpu, path):
    g = json.load(open(path))
    rec = MG.run_case(g["case"], "ours")
    for i, (a, b) in enumerate(zip(rec["per_frame"], g["per_frame"])):
        assert a == b, f"picture {i}: {[k for k in a if a[k] != b[k]]}"
    assert rec["stream_sha256"] == g["stream_sha256"]
