"""ctypes bindings of libh261b.so (include/h261b.h, include/h261b_abi.h).

The library is built in-tree (``h261enc_cuda_b200/lib``) by ``make -C
h261enc_cuda_b200/csrc`` or ``__graft_entry__.build()``.  There is no Python
or CPU fallback: if the shared object is missing, loading raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_float, c_int8, c_int16, c_int32, c_int64,
                    c_uint8, c_uint64, c_void_p)

import numpy as np

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
# H261B_LIB=check loads the checking build (bounds checks in the encode
# kernel, lib/libh261b_check.so, `make -C h261enc_cuda_b200/csrc check`)
CORE_PATH = os.path.join(LIB_DIR, "libh261b_check.so" if os.environ.get("H261B_LIB") == "check" else "libh261b.so")
SYNTH_PATH = os.path.join(LIB_DIR, "libh261b_synth.so")

H261B_OK = 0
ERRORS = {-1: "ARG", -2: "CUDA", -3: "NOMEM", -4: "BUDGET", -5: "STATE", -6: "NO_DEVICE"}
ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_BUDGET, ERR_STATE, ERR_NO_DEVICE = -1, -2, -3, -4, -5, -6

FRAME_TYPE_INTRA, FRAME_TYPE_INTER = 0, 1
MB_TYPE_INTRA, MB_TYPE_INTER = 0, 2
MB_MC, MB_FILTER, MB_COEFF = 1, 2, 4

# ---- exported symbols of the reference boundary (src/gpu_device.h:7-32)
ABI_SYMBOLS = (
    "h261_gpu_init",
    "h261_gpu_device_init_textures",
    "h261_gpu_device_deinit_textures",
    "h261_gpu_device_set_current",
    "h261_gpu_device_set_current_chroma_cb",
    "h261_gpu_device_set_current_chroma_cr",
    "h261_gpu_device_set_reference",
    "h261_gpu_device_set_reference_chroma_cb",
    "h261_gpu_device_set_reference_chroma_cr",
    "h261_gpu_device_init_me",
    "h261_gpu_device_deinit_me",
    "h261_gpu_device_me",
    "h261_init_macroblocks",
    "h261_deinit_macroblocks",
    "h261_gpu_device_encode_macroblocks",
    "h261_gpu_device_decode_macroblocks",
)

# ---- the layout-compatible structs as numpy dtypes (for reading results)
ME_MB_DTYPE = np.dtype([("intra", "<i4"), ("zero", "<i4"), ("cost", "<i4"), ("fcost", "<i4"),
                        ("mvx", "i1"), ("mvy", "i1"), ("pad", "<i2")])
MD_DTYPE = np.dtype([("cost", "<i4"), ("qadj", "<i4"), ("type", "<i4"), ("flags", "<i4"),
                     ("mvx", "<i4"), ("mvy", "<i4")])
MB_DTYPE = np.dtype([("addr", "<i4"), ("type", "<i4"), ("flags", "<i4"), ("quant", "<i4"),
                     ("mv", "<i4", 2), ("cbp", "<i4"), ("tcoeff", "<i4", (6, 64)),
                     ("mb_x", "<i4"), ("mb_y", "<i4")])
PICTURE_DTYPE = np.dtype([("session_id", "<i4"), ("frame_index", "<i4"), ("bytes", "<i4"), ("status", "<i4"),
                          ("bits", "<u8")])
RESULT_DTYPE = np.dtype([("type", "<i2"), ("flags", "<i2"), ("quant", "i1"), ("cbp", "i1"),
                         ("mvx", "i1"), ("mvy", "i1"), ("cost", "<i4"), ("coef_bits", "<i4")])
assert ME_MB_DTYPE.itemsize == 20 and MD_DTYPE.itemsize == 24 and MB_DTYPE.itemsize == 1572
assert RESULT_DTYPE.itemsize == 16


class EngineConfig(Structure):
    _fields_ = [("device", c_int32), ("max_sessions", c_int32), ("hbm_budget_bytes", c_int64),
                ("me_mode", c_int32), ("fmad", c_int32), ("warps_per_cta", c_int32),
                ("max_ctas", c_int32), ("copy_threads", c_int32), ("levels_to_host", c_int32),
                ("bits_host_bytes", c_int64), ("use_graphs", c_int32), ("kernel_split", c_int32),
                ("tail_items", c_int32), ("staging", c_int32), ("reserved", c_int32)]


class LaunchPlan(Structure):
    _fields_ = [("warps_per_cta", c_int32), ("max_ctas", c_int32), ("kernel_split", c_int32),
                ("tail_items", c_int32), ("staging", c_int32), ("source", c_int32), ("tuning", c_int32),
                ("reserved", c_int32)]


class SessionConfig(Structure):
    _fields_ = [("width", c_int32), ("height", c_int32), ("quant", c_int32),
                ("intra_period", c_int32), ("denoise", c_int32), ("bitstream", c_int32),
                ("rate_control", c_int32), ("bitrate", c_int32), ("psnr", c_int32)]


class FrameResult(Structure):
    _fields_ = [("frame_index", c_int32), ("frame_type", c_int32), ("quant", c_int32),
                ("num_mb", c_int32), ("mbs", c_void_p), ("levels", POINTER(c_int8)),
                ("bits", c_void_p), ("bits_bytes", c_int32), ("bits_status", c_int32),
                ("ssd", ctypes.c_uint64 * 3), ("psnr", ctypes.c_double * 3)]


class StepTiming(Structure):
    _fields_ = [("step", c_int64), ("upload_ms", c_float), ("wait_ms", c_float), ("encode_ms", c_float),
                ("bitstream_ms", c_float), ("total_ms", c_float), ("reserved", c_float)]


class SynthParams(Structure):
    _fields_ = [("width", c_int32), ("height", c_int32), ("kind", c_int32), ("seed", c_uint64),
                ("n_objects", c_int32), ("obj_min", c_int32), ("obj_max", c_int32),
                ("obj_vmax", c_int32), ("pan_dx", c_int32), ("pan_dy", c_int32),
                ("pan_period", c_int32), ("pan_rand", c_int32), ("scene_cut", c_int32),
                ("noise_sigma16", c_int32), ("block_motion_max", c_int32)]


_core = None
_synth = None


def _need(path: str) -> None:
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build the encode core first "
                           "(make -C h261enc_cuda_b200/csrc, or __graft_entry__.build())")


def core() -> ctypes.CDLL:
    """The encode core (CUDA).  Raises if it was not built."""
    global _core
    if _core is None:
        _need(CORE_PATH)
        lib = ctypes.CDLL(CORE_PATH)
        lib.h261b_last_error.restype = c_char_p
        lib.h261b_version.restype = c_char_p
        lib.h261b_abi_last_status.restype = c_int32
        lib.h261b_engine_config_default.argtypes = [POINTER(EngineConfig)]
        lib.h261b_engine_create.argtypes = [POINTER(EngineConfig), POINTER(c_void_p)]
        lib.h261b_engine_destroy.argtypes = [c_void_p]
        lib.h261b_session_bytes.argtypes = [c_int32, c_int32]
        lib.h261b_session_bytes.restype = c_int64
        lib.h261b_session_open.argtypes = [c_void_p, POINTER(SessionConfig), POINTER(c_int32)]
        lib.h261b_session_close.argtypes = [c_void_p, c_int32]
        lib.h261b_engine_reserve.argtypes = [c_void_p, POINTER(SessionConfig), c_int32]
        lib.h261b_engine_wait_step.argtypes = [c_void_p, c_int64]
        lib.h261b_engine_reserve_step.argtypes = [c_void_p, POINTER(SessionConfig), c_int32]
        lib.h261b_session_submit.argtypes = [c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_int32]
        lib.h261b_session_submit_device.argtypes = [c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_int32]
        lib.h261b_engine_submit_device_batch.argtypes = [c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                                                         c_void_p]
        lib.h261b_measure_sad_peak.argtypes = [c_int32, POINTER(ctypes.c_double)]
        lib.h261b_session_input.argtypes = [c_void_p, c_int32, c_int32, POINTER(POINTER(c_uint8)),
                                            POINTER(POINTER(c_uint8)), POINTER(POINTER(c_uint8))]
        lib.h261b_engine_submit_batch.argtypes = [c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                                                  c_void_p]
        lib.h261b_engine_submit_batch_async.argtypes = lib.h261b_engine_submit_batch.argtypes
        lib.h261b_engine_graph_stats.argtypes = [c_void_p, POINTER(c_int64), POINTER(c_int64)]
        lib.h261b_engine_launch_shape.argtypes = [c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]
        lib.h261b_engine_plan.argtypes = [c_void_p, POINTER(LaunchPlan), c_int32, c_void_p, c_void_p,
                                          POINTER(c_int32)]
        lib.h261b_engine_step_timing.argtypes = [c_void_p, POINTER(StepTiming)]
        lib.h261b_engine_last_bits_ms.argtypes = [c_void_p, POINTER(c_float)]
        lib.h261b_engine_step_pictures.argtypes = [c_void_p, c_int32, c_void_p, POINTER(c_int32),
                                                   POINTER(c_void_p), POINTER(ctypes.c_int64)]
        lib.h261b_engine_step_bits.argtypes = [c_void_p, POINTER(ctypes.c_int64), POINTER(c_int32)]
        lib.h261b_session_config_bytes.argtypes = [POINTER(SessionConfig)]
        lib.h261b_session_config_bytes.restype = c_int64
        lib.h261b_session_bits_bytes.argtypes = [c_int32, c_int32]
        lib.h261b_session_bits_bytes.restype = c_int64
        lib.h261b_engine_last_copy_bytes.argtypes = [c_void_p, POINTER(ctypes.c_int64), POINTER(ctypes.c_int64)]
        lib.h261b_engine_inputs.argtypes = [c_void_p, c_int32, c_void_p, c_void_p, POINTER(c_void_p), c_void_p]
        lib.h261b_engine_step_records.argtypes = [c_void_p, POINTER(c_void_p), POINTER(ctypes.c_int64),
                                                  POINTER(ctypes.c_int64)]
        lib.h261b_engine_step.argtypes = [c_void_p]
        lib.h261b_engine_sync.argtypes = [c_void_p]
        lib.h261b_engine_wait_previous.argtypes = [c_void_p]
        lib.h261b_session_result.argtypes = [c_void_p, c_int32, POINTER(FrameResult)]
        lib.h261b_session_recon.argtypes = [c_void_p, c_int32, c_void_p, c_void_p, c_void_p]
        lib.h261b_result_to_abi.argtypes = [POINTER(FrameResult), c_int32, c_void_p]
        lib.h261b_engine_last_kernel_ms.argtypes = [c_void_p, POINTER(c_float)]
        lib.h261b_engine_stats.argtypes = [c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_int64)]
        # reference boundary
        lib.h261_gpu_device_init_textures.argtypes = [c_int32, c_int32]
        for n in ("h261_gpu_device_set_current", "h261_gpu_device_set_current_chroma_cb",
                  "h261_gpu_device_set_current_chroma_cr", "h261_gpu_device_set_reference",
                  "h261_gpu_device_set_reference_chroma_cb", "h261_gpu_device_set_reference_chroma_cr"):
            getattr(lib, n).argtypes = [c_void_p, c_int32, c_int32]
        lib.h261_gpu_device_init_me.argtypes = [POINTER(c_void_p), c_int32, c_int32]
        lib.h261_gpu_device_deinit_me.argtypes = [POINTER(c_void_p)]
        lib.h261_gpu_device_me.argtypes = [c_void_p]
        lib.h261_init_macroblocks.argtypes = [POINTER(c_void_p), c_int32, c_int32, c_int32]
        lib.h261_deinit_macroblocks.argtypes = [c_void_p]
        lib.h261_gpu_device_encode_macroblocks.argtypes = [c_void_p]
        lib.h261_gpu_device_decode_macroblocks.argtypes = [c_void_p]
        _core = lib
    return _core


def synth() -> ctypes.CDLL:
    """The synthetic source generator (plain C)."""
    global _synth
    if _synth is None:
        _need(SYNTH_PATH)
        lib = ctypes.CDLL(SYNTH_PATH)
        lib.h261b_synth_preset.argtypes = [c_int32, c_int32, c_int32, c_uint64, POINTER(SynthParams)]
        lib.h261b_synth_create.argtypes = [POINTER(SynthParams), POINTER(c_void_p)]
        lib.h261b_synth_next.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        lib.h261b_synth_destroy.argtypes = [c_void_p]
        _synth = lib
    return _synth


class H261Error(RuntimeError):
    """A failed library call; `status` is its H261B_ERR_* code."""

    def __init__(self, message: str, status: int = 0):
        super().__init__(message)
        self.status = status


def check(rc: int, what: str) -> int:
    if rc < 0:
        msg = core().h261b_last_error().decode(errors="replace")
        raise H261Error(f"{what} failed ({ERRORS.get(rc, rc)}): {msg}", rc)
    return rc


def ptr(a: np.ndarray) -> c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return c_void_p(a.ctypes.data)
