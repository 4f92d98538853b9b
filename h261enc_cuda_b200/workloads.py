"""Named encode workloads (seeded, synthetic).

batch64     64 independent streams in one frame-step: 40 QCIF + 24 CIF,
            lengths uniform in 30..300 pictures, fixed QUANT uniform in
            4..24, per-stream seeds for the pan-and-objects generator with
            pan speeds in [-4, 4]; a stream that ends is replaced by a new
            one in the same slot (it starts with an intra picture).
stress1024  1024 QCIF streams, 60 pictures, QUANT 12, per-16x16-block random
            motion in [-15, 15] plus noise (motion-search stress).

Pictures come from a short seeded clip per stream, played forwards then
backwards, so a long run needs no long clip and shows no cut.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import synth


@dataclass
class Stream:
    width: int
    height: int
    quant: int
    length: int
    seed: int
    preset: int

    @property
    def num_mb(self) -> int:
        return (self.width // 16) * (self.height // 16)


def batch64(seed: int = 20261203, rank: int = 0) -> list[Stream]:
    rng = np.random.default_rng(seed + 7919 * rank)
    out = []
    for i in range(64):
        w, h = (176, 144) if i < 40 else (352, 288)
        out.append(Stream(w, h, int(rng.integers(4, 25)), int(rng.integers(30, 301)),
                          int(rng.integers(1, 2 ** 62)), synth.PRESET_STREAM))
    return out


def stress1024(seed: int = 20261204, rank: int = 0) -> list[Stream]:
    rng = np.random.default_rng(seed + 7919 * rank)
    return [Stream(176, 144, 12, 60, int(rng.integers(1, 2 ** 62)), synth.PRESET_BLOCK_MOTION) for _ in range(1024)]


WORKLOADS = {"batch64": batch64, "stress1024": stress1024}


def clip_index(k: int, clip_len: int) -> int:
    """Picture k of an endless forwards-backwards playback of a clip."""
    if clip_len == 1:
        return 0
    period = 2 * clip_len - 2
    r = k % period
    return r if r < clip_len else period - r


def make_clip(s: Stream, clip_len: int) -> np.ndarray:
    return synth.clip(s.preset, s.width, s.height, s.seed, clip_len)
