"""The encode kernel computes the forward DCT's rounding in float alone
(fdct_round in h261enc_cuda_b200/csrc/kernels.cu), where the reference widens
to double (mbgpu_kernels.cuh:413-437).  That is bit-exact only because
floorf((float)((double)p + 0.49999)) == floorf(p + 0.49999f) for every
finite float p; tests/rounding_check.c checks every float of magnitude
below 2^24 (about ten seconds) and a sample above."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_fdct_rounding_identity_holds_for_every_float(tmp_path):
    exe = tmp_path / "rounding_check"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-o", str(exe),
                    os.path.join(ROOT, "tests", "rounding_check.c"), "-lm"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    checked, differing, first = out.stdout.split()
    assert out.returncode == 0 and int(differing) == 0, f"{differing} floats differ, first {first}"
    assert int(checked) > 2_500_000_000
