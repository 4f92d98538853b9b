"""The checking build (lib/libh261b_check.so: the encode kernel tests the
index of every global access that depends on a vector, a work item or a
picture size, and of the motion compensation's window reads) encodes
border-heavy content -- per-block random motion up to +-15, QCIF and CIF,
the reference search and the full search, intra refresh -- without a single
failed check, and bit-exact to the oracle.  Run in a child process, which
loads the checking library instead of the normal one."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import json, sys
import numpy as np
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + "/oracle")
import oracle as O
from h261enc_cuda_b200 import _lib, synth
from h261enc_cuda_b200.engine import Engine, debug_check_status
assert _lib.CORE_PATH.endswith("libh261b_check.so"), _lib.CORE_PATH
out = {"cases": 0}
for (w, h, me_mode, q, intra, preset, seed) in [(176, 144, 0, 12, 3, 3, 71), (352, 288, 0, 8, 0, 3, 72),
                                                 (176, 144, 1, 12, 0, 3, 73), (352, 288, 0, 4, 2, 1, 74)]:
    n = 4
    fr = synth.clip(preset, w, h, seed, n)
    want = O.encode_sequence(fr, w, h, q, intra_period=intra, me_mode=me_mode)
    with Engine(me_mode=me_mode, warps_per_cta=4) as e:
        sid = e.open(w, h, q, intra_period=intra)
        for i in range(n):
            e.submit_frame(sid, fr[i])
            e.step()
            e.sync()
            got = e.result(sid).to_abi(w)
            assert np.array_equal(got["tcoeff"], want["mbs"][i]["tcoeff"]), (w, me_mode, i)
            assert np.array_equal(got["mv"], want["mbs"][i]["mv"]), (w, me_mode, i)
            assert np.array_equal(np.concatenate(e.recon(sid)), want["recon"][i]), (w, me_mode, i)
    out["cases"] += 1
en, n, site, val = debug_check_status()
out.update(enabled=en, violations=n, site=site, value=val)
print(json.dumps(out))
'''


@pytest.mark.gpu
def test_checking_build_encodes_without_a_failed_check(gpu):
    lib = os.path.join(ROOT, "h261enc_cuda_b200", "lib", "libh261b_check.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "h261enc_cuda_b200", "csrc"), "check"], check=True)
    env = dict(os.environ, H261B_LIB="check")
    r = subprocess.run([sys.executable, "-c", f"ROOT = {ROOT!r}\n" + CHILD], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["cases"] == 4
    assert res["enabled"], "the child did not load the checking build"
    assert res["violations"] == 0, f"failed checks: {res}"


def test_normal_build_reports_checks_disabled():
    from h261enc_cuda_b200 import _lib
    if os.environ.get("H261B_LIB") == "check":
        pytest.skip("this process loaded the checking build")
    from h261enc_cuda_b200.engine import debug_check_status
    assert _lib.core() is not None
    en, n, _, _ = debug_check_status()
    assert not en and n == 0
