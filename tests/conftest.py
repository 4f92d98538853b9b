import ctypes
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built sm_100a library")


def _cuda_devices() -> int:
    for name in ("libcuda.so.1", "libcuda.so"):
        try:
            lib = ctypes.CDLL(name)
        except OSError:
            continue
        if lib.cuInit(0) != 0:
            return 0
        n = ctypes.c_int(0)
        if lib.cuDeviceGetCount(ctypes.byref(n)) != 0:
            return 0
        return n.value
    return 0


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and the core if a checkout lacks them."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    lib = os.path.join(ROOT, "h261enc_cuda_b200", "lib")
    if not (os.path.exists(os.path.join(lib, "libh261b.so")) and os.path.exists(os.path.join(lib, "libh261b_synth.so"))):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "h261enc_cuda_b200", "csrc")], check=True)


@pytest.fixture(scope="session")
def gpu():
    if _cuda_devices() < 1:
        pytest.fail("a GPU test ran without a visible CUDA device")
    return True
