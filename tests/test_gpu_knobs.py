"""Every launch plan of the encode kernel writes the same bytes: the fused
kernel and the split search + encode kernels (chained by a programmatic
dependent launch, or with the device rate control between them), CTA widths,
tail lengths, and the two ways of staging the search window (16-byte
cp.async copies, or one bulk copy per row completed on a shared-memory
barrier).  A mixed batch -- QCIF and CIF, fixed QUANT and CBR rate control,
sessions joining late -- equals the oracle's frame loop picture by picture,
and no bulk-staging wait gives up.  The tuner then picks a plan on live
steps and reports what it measured."""
import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import synth
from h261enc_cuda_b200.engine import Engine, stage_timeouts

pytestmark = pytest.mark.gpu

# (w, h, quant (0: CBR), bitrate, first step, seed)
SPECS = [(176, 144, 8, 0, 0, 301), (352, 288, 12, 0, 0, 302), (176, 144, 0, 128000, 0, 303),
         (352, 288, 0, 1000000, 1, 304), (176, 144, 20, 0, 2, 305), (352, 288, 5, 0, 0, 306)]
N = 5
_want = {}


def _clips():
    return [synth.clip(2 if k % 2 else 3, w, h, seed, N) for k, (w, h, q, br, start, seed) in enumerate(SPECS)]


def _oracle(me_mode):
    if me_mode not in _want:
        clips = _clips()
        _want[me_mode] = [O.encode_stream(c, w, h, quant=q, bitrate=br or 384000, me_mode=me_mode)
                          for c, (w, h, q, br, start, seed) in zip(clips, SPECS)]
    return _want[me_mode]


def _run(me_mode, **knobs):
    clips = _clips()
    got = [[] for _ in SPECS]
    with Engine(me_mode=me_mode, levels_to_host=0, **knobs) as e:
        sids = [None] * len(SPECS)
        for t in range(N + 2):
            for k, (w, h, q, br, start, seed) in enumerate(SPECS):
                i = t - start
                if i == 0:
                    sids[k] = (e.open(w, h, q, bitstream=1) if q else
                               e.open(w, h, 10, bitstream=1, rate_control=1, bitrate=br))
                if 0 <= i < N:
                    e.submit_frame(sids[k], clips[k][i])
            e.step()
            e.sync()
            for k, (w, h, q, br, start, seed) in enumerate(SPECS):
                if 0 <= t - start < N:
                    r = e.result(sids[k])
                    got[k].append((r.bits, r.quant, np.concatenate(e.recon(sids[k]))))
        plan, log = e.plan()
    return got, plan, log


def _check(got, want, where):
    for k, (bits, nb, nq, rec) in enumerate(want):
        off = 0
        for i in range(N):
            b, q, r = got[k][i]
            assert q == nq[i], f"{where}: session {k} picture {i}: QUANT"
            assert b == bits[off:off + nb[i]], f"{where}: session {k} picture {i}: bytes"
            assert np.array_equal(r, rec[i]), f"{where}: session {k} picture {i}: reconstruction"
            off += nb[i]


@pytest.mark.parametrize("me_mode,warps,split,tail,staging", [
    (0, 4, 1, 3, 1),     # fused kernel, cp.async staging (the plan of the first version)
    (0, 4, 2, 3, 1),     # search kernel + encode kernel
    (0, 8, 2, 3, 2),     # split, bulk row copies
    (0, 2, 1, 1, 2),     # fused, bulk, no tail draws
    (0, 8, 1, 5, 1),     # fused, four tail draws per warp
    (1, 4, 2, 3, 2),     # full search, split, bulk
])
def test_every_plan_matches_oracle(gpu, me_mode, warps, split, tail, staging):
    stage_timeouts()
    got, plan, _ = _run(me_mode, warps_per_cta=warps, kernel_split=split, tail_items=tail, staging=staging)
    assert (plan["warps_per_cta"], plan["kernel_split"], plan["tail_items"], plan["staging"]) == \
        (warps, split, tail, staging)
    assert plan["source"] == 0
    _check(got, _oracle(me_mode), f"plan {(warps, split, tail, staging)}")
    assert stage_timeouts() == 0


TUNER_CHILD = r'''
import json, sys
import numpy as np
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + "/oracle")
import oracle as O
from h261enc_cuda_b200 import synth
from h261enc_cuda_b200.engine import Engine
n, specs = 40, [(176, 144, 8, 401), (352, 288, 12, 402), (176, 144, 16, 403)]
clips = [synth.clip(2, w, h, seed, n) for (w, h, q, seed) in specs]
bits = [b"" for _ in specs]
with Engine(levels_to_host=0) as e:
    sids = [e.open(w, h, q, bitstream=1) for (w, h, q, seed) in specs]
    for i in range(n):
        e.submit_frames(sids, [c[i] for c in clips])
        e.step()
        e.sync()
        for k, sid in enumerate(sids):
            bits[k] += e.result(sid).bits
    plan, log = e.plan()
ok = all(bits[k] == O.encode_stream(clips[k], w, h, quant=q)[0] for k, (w, h, q, seed) in enumerate(specs))
print(json.dumps({"plan": plan, "log": log, "bitexact": ok}))
'''


def test_tuner_measures_every_knob(gpu):
    """In a fresh process (the tuning of a device is kept for the rest of a
    process), an engine with every knob left open tunes on its first
    mostly-inter steps: the CTA widths of the fused and the split kernels,
    then tail lengths and both staging variants on the winner; the output
    is the oracle's throughout."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", f"ROOT = {root!r}\n" + TUNER_CHILD], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["bitexact"], "a tuning step changed the output"
    plan, log = res["plan"], res["log"]
    assert plan["source"] == 1 and plan["tuning"] == 0, plan
    assert {p["kernel_split"] for p, _ in log} == {1, 2}, log
    assert {p["staging"] for p, _ in log} == {1, 2}, log
    assert {p["tail_items"] for p, _ in log} >= {1, 3, 5}, log
    # three rounds of every candidate: 5 in stage 1, 4 in stage 2
    assert len(log) == 27, log
    assert all(ms > 0 for _, ms in log)
