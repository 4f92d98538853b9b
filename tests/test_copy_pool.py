"""The staging copy pool on the CPU (h261enc_cuda_b200/csrc/copy_pool.h, built
with g++): the batches of h261b_engine_submit_batch (synchronous) and
h261b_engine_submit_batch_async (started, then joined by the next step) land
byte for byte, with 0 to 7 workers and pieces split across plane copies; and
with failures injected on the host -- workers the system cannot start
(the pool keeps the ones that started, down to none) and a worker that
stalls in the middle of a batch (the others and the caller take the rest,
and no call returns before every byte is in place)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_copy_pool_batches_land(tmp_path):
    exe = tmp_path / "copy_pool_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", os.path.join(ROOT, "h261enc_cuda_b200", "csrc"),
                    "-o", str(exe), os.path.join(ROOT, "tests", "copy_pool_check.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok"
