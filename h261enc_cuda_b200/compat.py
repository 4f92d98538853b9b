"""The reference's device boundary (src/gpu_device.h:7-32) from Python.

``Boundary`` drives the sixteen entry points of libh261b.so exactly the way
the reference's host code does (src/h261_main.c:319-365): upload current and
reference planes, run motion estimation, let the caller decide modes and
QUANT, encode, decode.  ctypes mirrors of the reference structs give access
to the library-owned result arrays.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, Structure, c_int32, c_uint8, c_void_p

import numpy as np

from . import _lib


class MeGpu(Structure):  # me_gpu_t, src/h261_types.h:61-79
    _fields_ = [("i_mb_width", c_int32), ("i_mb_height", c_int32), ("i_num_mb", c_int32),
                ("prgs_macroblocks_device", c_void_p), ("prgs_macroblocks_result", c_void_p),
                ("ps_candidate_vector_device", c_void_p), ("ps_candidate_vector_host", c_void_p),
                ("ps_starting_vector_device", c_void_p), ("ps_starting_vector_host", c_void_p),
                ("pi8_motion_vector_limits_device", c_void_p), ("pi8_motion_vector_limits_host", c_void_p),
                ("p_cuda", c_void_p)]


class Macroblocks(Structure):  # h261_macroblocks_t, src/h261_types.h:152-192
    _fields_ = [("i_mb_width", c_int32), ("i_mb_height", c_int32), ("i_num_mb", c_int32),
                ("ps_macroblocks", c_void_p), ("ps_macroblocks_device", c_void_p),
                ("ps_denoise_host", c_void_p), ("ps_denoise_device", c_void_p),
                ("pi_mb_types_host", c_void_p), ("pi_mb_types_device", c_void_p),
                ("pi_mb_flags_host", c_void_p), ("pi_mb_flags_device", c_void_p),
                ("pi_mb_quant_host", c_void_p), ("pi_mb_quant_device", c_void_p),
                ("pi_mb_mv_x_host", c_void_p), ("pi_mb_mv_x_device", c_void_p),
                ("pi_mb_mv_y_host", c_void_p), ("pi_mb_mv_y_device", c_void_p),
                ("pui8_reconstructed_Y_device", c_void_p), ("pui8_reconstructed_Y_host", c_void_p),
                ("pui8_reconstructed_Cr_device", c_void_p), ("pui8_reconstructed_Cr_host", c_void_p),
                ("pui8_reconstructed_Cb_device", c_void_p), ("pui8_reconstructed_Cb_host", c_void_p),
                ("i_num_blocks", c_int32), ("i_num_coeff_blocks", c_int32),
                ("pi_coeff_blocks_device", c_void_p), ("pi_coeff_blocks_host", c_void_p),
                ("p_cuda", c_void_p)]


class ModeDecision(Structure):  # h261_mode_decision_t, src/h261_types.h:92-96
    _fields_ = [("i_mb_width", c_int32), ("i_mb_height", c_int32), ("prgs_mb", c_void_p)]


class Frame(Structure):  # h261_frame_t
    _fields_ = [("i_width", c_int32), ("i_height", c_int32), ("i_stride_y", c_int32), ("i_stride_c", c_int32),
                ("pui8_Y", c_void_p), ("pui8_Cr", c_void_p), ("pui8_Cb", c_void_p)]


class Picture(Structure):  # h261_picture_t
    _fields_ = [("i_picture_start_code", c_int32), ("i_temporal_reference", c_int32),
                ("i_split_screen_indicator", c_int32), ("i_document_camera_indicator", c_int32),
                ("i_freeze_picture_release", c_int32), ("i_source_format", c_int32),
                ("i_highres_mode", c_int32), ("i_spare_bit", c_int32),
                ("i_num_extra_insertion_information", c_int32), ("rgui8_extra", c_uint8 * 1),
                ("gob", c_int32 * 8), ("i_quantiser", c_int32), ("i_frame_type", c_int32)]


class Context(Structure):  # h261_context_t, src/h261_types.h:267-284
    _fields_ = [("i_source_format", c_int32), ("i_frame_counter", c_int32),
                ("s_current_frame", Frame), ("s_reference_frame", Frame), ("s_picture", Picture),
                ("s_bitstream", c_int32 * 6), ("ps_mode_decision", POINTER(ModeDecision)),
                ("s_ratectrl", c_int32 * 10), ("ps_macroblocks", POINTER(Macroblocks))]


assert ctypes.sizeof(MeGpu) == 88 and ctypes.sizeof(Macroblocks) == 208
assert ctypes.sizeof(Picture) == 80 and ctypes.sizeof(Context) == 248
assert Context.ps_mode_decision.offset == 192 and Context.ps_macroblocks.offset == 240


class Boundary:
    """One process-global encoder through the reference's sixteen calls."""

    def __init__(self, width: int, height: int, denoise: int = 5):
        self.lib = lib = _lib.core()
        self.w, self.h = width, height
        lib.h261_gpu_init()
        lib.h261_gpu_device_init_textures(width, height)
        self._mbs = c_void_p()
        lib.h261_init_macroblocks(ctypes.byref(self._mbs), width, height, denoise)
        self._me = c_void_p()
        lib.h261_gpu_device_init_me(ctypes.byref(self._me), width, height)
        self._check("init")
        self.me = ctypes.cast(self._me, POINTER(MeGpu)).contents
        self.mbs = ctypes.cast(self._mbs, POINTER(Macroblocks)).contents
        self.nmb = self.me.i_num_mb
        self._md_arr = np.zeros(self.nmb, _lib.MD_DTYPE)
        self._md = ModeDecision(width // 16, height // 16, self._md_arr.ctypes.data)
        self._ctx = Context()
        self._ctx.ps_mode_decision = ctypes.pointer(self._md)
        self._ctx.ps_macroblocks = ctypes.cast(self._mbs, POINTER(Macroblocks))

    def _check(self, what: str) -> None:
        st = self.lib.h261b_abi_last_status()
        if st != 0:
            raise _lib.H261Error(f"{what}: {self.lib.h261b_last_error().decode(errors='replace')}")

    def set_current(self, y, cb, cr) -> None:
        w, h = self.w, self.h
        self.lib.h261_gpu_device_set_current(_lib.ptr(y), w, h)
        self.lib.h261_gpu_device_set_current_chroma_cb(_lib.ptr(cb), w // 2, h // 2)
        self.lib.h261_gpu_device_set_current_chroma_cr(_lib.ptr(cr), w // 2, h // 2)
        self._check("set_current")

    def set_reference(self, y, cb, cr) -> None:
        w, h = self.w, self.h
        self.lib.h261_gpu_device_set_reference(_lib.ptr(y), w, h)
        self.lib.h261_gpu_device_set_reference_chroma_cb(_lib.ptr(cb), w // 2, h // 2)
        self.lib.h261_gpu_device_set_reference_chroma_cr(_lib.ptr(cr), w // 2, h // 2)
        self._check("set_reference")

    def motion_estimation(self) -> np.ndarray:
        self.lib.h261_gpu_device_me(self._me)
        self._check("h261_gpu_device_me")
        buf = (c_uint8 * (20 * self.nmb)).from_address(self.me.prgs_macroblocks_result)
        return np.frombuffer(buf, _lib.ME_MB_DTYPE).copy()

    def encode(self, md: np.ndarray, quant: int, frame_type: int) -> np.ndarray:
        self._md_arr[:] = md
        self._ctx.s_picture.i_quantiser = quant
        self._ctx.s_picture.i_frame_type = frame_type
        self.lib.h261_gpu_device_encode_macroblocks(ctypes.byref(self._ctx))
        self._check("h261_gpu_device_encode_macroblocks")
        buf = (c_uint8 * (1572 * self.nmb)).from_address(self.mbs.ps_macroblocks)
        return np.frombuffer(buf, _lib.MB_DTYPE).copy()

    def decode(self):
        self.lib.h261_gpu_device_decode_macroblocks(ctypes.byref(self._ctx))
        self._check("h261_gpu_device_decode_macroblocks")
        ny, nc = self.w * self.h, self.w * self.h // 4
        y = np.frombuffer((c_uint8 * ny).from_address(self.mbs.pui8_reconstructed_Y_host), np.uint8).copy()
        cb = np.frombuffer((c_uint8 * nc).from_address(self.mbs.pui8_reconstructed_Cb_host), np.uint8).copy()
        cr = np.frombuffer((c_uint8 * nc).from_address(self.mbs.pui8_reconstructed_Cr_host), np.uint8).copy()
        return y, cb, cr

    def close(self) -> None:
        if self._me:
            self.lib.h261_gpu_device_deinit_me(ctypes.byref(self._me))
            self.lib.h261_deinit_macroblocks(self._mbs)
            self.lib.h261_gpu_device_deinit_textures()
            self._me = c_void_p()
