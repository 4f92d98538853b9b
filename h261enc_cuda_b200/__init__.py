"""h261enc_cuda_b200 -- a B200 (sm_100a) H.261 encode core.

The product is ``lib/libh261b.so``: hand-written CUDA kernels for motion
estimation, mode decision, motion compensation with the loop filter, DCT,
denoise, quantisation and reconstruction, exported through the reference
encoder's own ``gpu_device.h`` boundary (``include/h261b_abi.h``) and through
a batched multi-session engine (``include/h261b.h``).  This package holds
the ctypes bindings and the host-side helpers around it; it never falls back
to a CPU path.
"""
from . import _lib
from ._lib import ABI_SYMBOLS, H261Error, core, synth as synth_lib

__all__ = ["ABI_SYMBOLS", "H261Error", "core", "synth_lib"]
