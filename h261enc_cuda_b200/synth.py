"""Seeded synthetic YUV 4:2:0 sources (wrapper of libh261b_synth.so).

The reference ships no test material; the workloads the encoder is checked
and measured on are generated from seeds (see include/h261b_synth.h for the
content model).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

PRESET_PAN = 0          # QCIF-style pan + two moving rectangles
PRESET_CIF_SCENES = 1   # pan redrawn every 30 frames, 6 objects, scene cut
PRESET_STREAM = 2       # per-stream variant of 0, pan speed from the seed
PRESET_BLOCK_MOTION = 3  # per-16x16-block random motion


class Source:
    """An endless seeded picture source: ``next()`` returns (y, cb, cr)."""

    def __init__(self, preset: int, width: int, height: int, seed: int):
        lib = _lib.synth()
        self.width, self.height = width, height
        self.params = _lib.SynthParams()
        if lib.h261b_synth_preset(preset, width, height, ctypes.c_uint64(seed), ctypes.byref(self.params)):
            raise ValueError(f"unknown preset {preset}")
        h = ctypes.c_void_p()
        if lib.h261b_synth_create(ctypes.byref(self.params), ctypes.byref(h)):
            raise ValueError(f"cannot create a {width}x{height} source")
        self._h = h
        self.frames = 0

    def next_into(self, y: np.ndarray, cb: np.ndarray, cr: np.ndarray) -> int:
        assert y.size == self.width * self.height and cb.size == cr.size == y.size // 4
        self.frames += 1
        return _lib.synth().h261b_synth_next(self._h, _lib.ptr(y), _lib.ptr(cb), _lib.ptr(cr))

    def next(self):
        y = np.empty(self.width * self.height, np.uint8)
        cb = np.empty(y.size // 4, np.uint8)
        cr = np.empty(y.size // 4, np.uint8)
        self.next_into(y, cb, cr)
        return y, cb, cr

    def clip(self, n: int) -> np.ndarray:
        """n frames as one packed array (n, W*H*3/2), Y then Cb then Cr."""
        fs = self.width * self.height
        out = np.empty((n, fs * 3 // 2), np.uint8)
        for i in range(n):
            self.next_into(out[i, :fs], out[i, fs:fs + fs // 4], out[i, fs + fs // 4:])
        return out

    def close(self) -> None:
        if self._h:
            _lib.synth().h261b_synth_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def clip(preset: int, width: int, height: int, seed: int, frames: int) -> np.ndarray:
    s = Source(preset, width, height, seed)
    try:
        return s.clip(frames)
    finally:
        s.close()


def split(frame: np.ndarray, width: int, height: int):
    """(y, cb, cr) views of one packed frame."""
    fs = width * height
    return frame[:fs], frame[fs:fs + fs // 4], frame[fs + fs // 4:fs + fs // 2]
