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


TIMEOUT_CHILD = r'''
import json, os, sys
import numpy as np
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + "/oracle")
import oracle as O
from h261enc_cuda_b200 import synth
from h261enc_cuda_b200.engine import Engine, stage_timeouts
w, h, n = 176, 144, 3
fr = synth.clip(0, w, h, 81, n)
want = O.encode_sequence(fr, w, h, 8)

def encode():
    with Engine(warps_per_cta=4, kernel_split=1, tail_items=3, staging=2) as e:
        sid = e.open(w, h, 8)
        ok = True
        for i in range(n):
            e.submit_frame(sid, fr[i])
            e.step()
            e.sync()
            ok = ok and np.array_equal(e.result(sid).to_abi(w)["tcoeff"], want["mbs"][i]["tcoeff"])
            ok = ok and np.array_equal(np.concatenate(e.recon(sid)), want["recon"][i])
    return ok

stage_timeouts()
forced = encode()                       # every warp's first wait runs out
t_forced = stage_timeouts()
del os.environ["H261B_TEST_STAGE_SHORT"]
normal = encode()                       # a new engine in the same context
t_normal = stage_timeouts()
print(json.dumps({"forced_ok": bool(forced), "forced_timeouts": t_forced, "normal_ok": bool(normal),
                  "normal_timeouts": t_normal}))
'''


@pytest.mark.gpu
def test_bounded_staging_wait_runs_out_and_reports(gpu):
    """The bulk staging's wait is bounded.  The checking build can make
    every warp's first staging announce 16 bytes more than its copies bring
    (H261B_TEST_STAGE_SHORT), so that the wait runs out: the kernel counts it
    (h261b_stage_status), stops using that barrier, finishes with the data
    the copies did bring -- the output is still the oracle's -- and the
    context stays usable: a new engine in the same process encodes with no
    wait running out.  No fault and no hang is made; the failure is an
    announcement that never completes."""
    lib = os.path.join(ROOT, "h261enc_cuda_b200", "lib", "libh261b_check.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "h261enc_cuda_b200", "csrc"), "check"], check=True)
    env = dict(os.environ, H261B_LIB="check", H261B_TEST_STAGE_SHORT="1")
    r = subprocess.run([sys.executable, "-c", f"ROOT = {ROOT!r}\n" + TIMEOUT_CHILD], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["forced_timeouts"] > 0, res
    assert res["forced_ok"], "the output changed when the staging wait ran out"
    assert res["normal_timeouts"] == 0 and res["normal_ok"], res


CODES_WAIT_CHILD = r'''
import json, os, sys
import numpy as np
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + "/oracle")
import oracle as O
from h261enc_cuda_b200 import synth
from h261enc_cuda_b200.engine import Engine
w, h, n = 176, 144, 3
fr = synth.clip(2, w, h, 83, n)
want = O.encode_sequence(fr, w, h, 8)

def encode():
    out = []
    with Engine(warps_per_cta=4, kernel_split=1, tail_items=3, staging=1, levels_to_host=1) as e:
        sid = e.open(w, h, 8, bitstream=1)
        for i in range(n):
            e.submit_frame(sid, fr[i])
            e.step()
            e.sync()
            r = e.result(sid)
            same = (np.array_equal(r.to_abi(w)["tcoeff"], want["mbs"][i]["tcoeff"]) and
                    np.array_equal(np.concatenate(e.recon(sid)), want["recon"][i]))
            wrote = O.write_picture_oracle(r.to_abi(w), w, h, i, r.frame_type, 8)
            out.append({"status": int(r.bits_status), "same": bool(same),
                        "bits_ok": r.bits is not None and r.bits == wrote})
    return out

forced = encode()                       # every codes warp's wait runs out
del os.environ["H261B_TEST_CODES_WAIT"]
normal = encode()                       # a new engine in the same context
print(json.dumps({"forced": forced, "normal": normal}))
'''


@pytest.mark.gpu
def test_bounded_codes_wait_runs_out_and_refuses(gpu):
    """The codes kernel waits, bounded, for each picture's MBs to be counted
    done by the encode launch.  The checking build can make it wait for one
    MB more than the picture has (H261B_TEST_CODES_WAIT), for 2 ms: the wait
    runs out, the step is marked and the layout refuses its pictures (a
    negative bitstream status), while the records and reconstructions are
    still the oracle's; a new engine in the same process then writes every
    picture's bitstream as the oracle's writer does.  No fault and no hang
    is made; the failure is a count that never completes."""
    lib = os.path.join(ROOT, "h261enc_cuda_b200", "lib", "libh261b_check.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "h261enc_cuda_b200", "csrc"), "check"], check=True)
    env = dict(os.environ, H261B_LIB="check", H261B_TEST_CODES_WAIT="1")
    r = subprocess.run([sys.executable, "-c", f"ROOT = {ROOT!r}\n" + CODES_WAIT_CHILD], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert all(p["status"] < 0 and p["same"] for p in res["forced"]), res
    assert all(p["status"] == 0 and p["same"] and p["bits_ok"] for p in res["normal"]), res
