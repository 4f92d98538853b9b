"""Serving: encode sessions that arrive over time, admitted under an HBM
budget and batched continuously on one device.

A request is one encode session (picture size, QUANT, number of pictures).
Its pictures are released at a fixed rate (30 per second) from the moment it
is admitted.  The loop:

* takes arrivals, and admits waiting requests in arrival order while the
  engine's HBM budget accepts them (``h261b_session_open`` refuses with
  H261B_ERR_BUDGET beyond it; a refused request waits for sessions to end);
* every iteration queues the picture of every admitted session whose
  release time has come (continuous batching: a session admitted while
  others are on the GPU joins the next step), copies them on the engine's
  threads while the previous step is read, and issues one step;
* reads each step's bitstreams one step later (a picture that did not fit
  the host arena is read from the device) and records, per picture, the
  latency from its release to its bitstream on the host;
* closes a session once its last picture has been read.

Pictures come from a shared pool of synthetic clips (a session reads its clip
forwards and backwards), so that memory does not grow with the number of
sessions.  The encoder treats every session independently, so each result is
what the session produces alone (tests/test_gpu_serving.py checks it).
"""
from __future__ import annotations

import ctypes
import gc
import heapq
import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import synth
from ._lib import ERR_BUDGET, H261Error


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start
    width: int
    height: int
    quant: int
    frames: int
    seed: int


def poisson_requests(rate: float, duration: float, seed: int = 0, cif_share: float = 0.3,
                     frames=(30, 600), quant=(4, 24)) -> List[Request]:
    """Arrivals of a Poisson process of `rate` sessions per second over
    `duration` seconds: 70 % QCIF / 30 % CIF, length and QUANT uniform."""
    rng = np.random.default_rng(seed)
    out, t, rid = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        cif = rng.random() < cif_share
        out.append(Request(rid, t, 352 if cif else 176, 288 if cif else 144, int(rng.integers(quant[0], quant[1] + 1)),
                           int(rng.integers(frames[0], frames[1] + 1)), int(rng.integers(1 << 31))))
        rid += 1


class ClipPool:
    """A few synthetic clips per picture size, shared by all sessions."""

    def __init__(self, clips_per_size: int = 8, length: int = 30, seed: int = 1000):
        self.length = length
        self.clips = {}
        for (w, h) in ((176, 144), (352, 288)):
            self.clips[(w, h)] = [synth.clip(2, w, h, seed + k, length) for k in range(clips_per_size)]

    def frame(self, width: int, height: int, seed: int, index: int) -> np.ndarray:
        pool = self.clips[(width, height)]
        clip = pool[seed % len(pool)]
        period = 2 * self.length - 2
        j = index % period
        return clip[j if j < self.length else period - j]


@dataclass
class _Live:
    req: Request
    sid: int
    start: float            # admission time: picture j is released at start + j / fps
    queued: int = 0         # pictures queued so far
    done: int = 0           # pictures read back
    bits: Optional[List[bytes]] = None


@dataclass
class ServeStats:
    duration: float
    pictures: int
    macroblocks: int
    steps: int
    admitted: int
    refused_at_least_once: int
    max_concurrent: int
    max_session_bytes: int
    latencies_ms: np.ndarray = field(repr=False, default=None)
    released_s: np.ndarray = field(repr=False, default=None)   # each picture's release time

    def summary(self) -> dict:
        lat = self.latencies_ms
        late = lat[self.released_s >= self.duration / 2] if self.released_s is not None else lat[:0]
        return {
            "duration_s": self.duration, "pictures": self.pictures, "mb_per_s": self.macroblocks / self.duration,
            "steps": self.steps, "pictures_per_step": self.pictures / max(self.steps, 1),
            "sessions_admitted": self.admitted, "sessions_waited_for_budget": self.refused_at_least_once,
            "max_concurrent_sessions": self.max_concurrent, "max_session_bytes": self.max_session_bytes,
            "latency_ms": {"p50": float(np.percentile(lat, 50)) if lat.size else None,
                           "p99": float(np.percentile(lat, 99)) if lat.size else None,
                           "max": float(lat.max()) if lat.size else None},
            "latency_ms_second_half": {"p50": float(np.percentile(late, 50)) if late.size else None,
                                       "p99": float(np.percentile(late, 99)) if late.size else None,
                                       "max": float(late.max()) if late.size else None},
        }


def expected_concurrency(rate: float, mean_frames: float, fps: float, share: float, margin: float = 1.25) -> int:
    """Sessions of one kind open at once in steady state (Little's law:
    arrival rate x time in the system), with a margin: the capacity a server
    plans for a Poisson stream of known rate and length distribution."""
    return int(math.ceil(rate * share * mean_frames / fps * margin))


class Server:
    """The request loop around one engine (which must have been created
    with the HBM budget that admission obeys)."""

    def __init__(self, engine, pool: ClipPool, fps: float = 30.0, keep_bits_for=()):
        self.e = engine
        self.pool = pool
        self.fps = fps
        self.keep = set(keep_bits_for)      # request ids whose bitstreams are kept (tests)
        self.bits: Dict[int, List[bytes]] = {}

    def plan(self, capacity: Dict[tuple, int], burst: float = 0.5) -> None:
        """Allocate the device blocks of {(width, height): sessions} up front,
        so that admissions during the run take pooled blocks, and size the
        step arenas for a step holding `burst` of those sessions' pictures
        (what piles up if the loop falls behind by burst / fps seconds)."""
        for (w, h), n in capacity.items():
            self.e.reserve(w, h, n, bitstream=1)
            self.e.reserve_step(w, h, int(math.ceil(n * burst)))

    def run(self, requests: List[Request], duration: float, drain: bool = False,
            clock=time.perf_counter) -> ServeStats:
        """Serve `requests` (arrival times within `duration` seconds).  The
        statistics cover [0, duration]; with drain=True the sessions still
        running then are encoded to their end first, else they are closed.

        Python's cyclic garbage collector is off while the loop runs: its
        full passes paused the loop for 40-70 ms, long enough for a step's
        worth of pictures from every session to pile up behind it.  The
        loop's objects hold no reference cycles, so reference counting
        frees them all."""
        enabled = gc.isenabled()
        gc.collect()
        gc.disable()
        try:
            return self._run(requests, duration, drain, clock)
        finally:
            if enabled:
                gc.enable()

    def _run(self, requests, duration, drain, clock) -> ServeStats:
        e, fps = self.e, self.fps
        arrivals = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: deque = deque()
        live: Dict[int, _Live] = {}          # by session id
        due: list = []                       # heap of (release time, session id), one entry per session
        in_step: Dict[int, list] = {}        # step number -> [(session id, release time)]
        lat: List[float] = []
        rel: List[float] = []
        refused = set()
        st = {"pictures": 0, "mbs": 0, "bytes": 0, "max_bytes": 0}
        steps = admitted = max_live = 0
        t0 = clock()

        def close(sid: int) -> None:
            s = live.pop(sid)
            if s.bits is not None:
                self.bits[s.req.rid] = s.bits
            e.close(sid)
            st["bytes"] -= self._bytes(s.req)

        def read_step(k: int) -> None:
            pics, _ = e.step_pictures(len(in_step[k]) + 8)
            got = {int(p["session_id"]): p for p in pics}
            now = clock() - t0
            for sid, release in in_step.pop(k):
                s, p = live[sid], got[sid]
                if p["status"] == 1:
                    # the picture did not fit the host arena (the engine
                    # grows it for later steps): read it from the device
                    bits = e.result(sid, copy=False).bits
                    if bits is None:
                        raise RuntimeError(f"session {s.req.rid}: picture {s.done} has no bitstream")
                elif p["status"] != 0:
                    raise RuntimeError(f"session {s.req.rid}: picture {s.done} has no bitstream")
                else:
                    bits = None
                if s.bits is not None:
                    s.bits.append(bits if bits is not None else ctypes.string_at(int(p["bits"]), int(p["bytes"])))
                s.done += 1
                if now <= duration or drain:
                    lat.append((now - release) * 1e3)
                    rel.append(release)
                    st["pictures"] += 1
                    st["mbs"] += (s.req.width // 16) * (s.req.height // 16)
                if s.done == s.req.frames:
                    close(sid)

        step_no, prev = 0, None
        while True:
            now = clock() - t0
            stopping = now >= duration and not drain
            if not stopping:
                while arrivals and arrivals[0].arrival <= now:
                    waiting.append(arrivals.popleft())
                # admission in arrival order while the HBM budget holds
                while waiting:
                    r = waiting[0]
                    try:
                        sid = e.open(r.width, r.height, r.quant, bitstream=1)
                    except H261Error as err:
                        if err.status != ERR_BUDGET:
                            raise
                        refused.add(r.rid)
                        break
                    waiting.popleft()
                    live[sid] = _Live(r, sid, now, bits=[] if r.rid in self.keep else None)
                    heapq.heappush(due, (now, sid))
                    admitted += 1
                    st["bytes"] += self._bytes(r)
                    st["max_bytes"] = max(st["max_bytes"], st["bytes"])
                max_live = max(max_live, len(live))
            # the released picture of every session whose picture is due
            batch = []
            while due and due[0][0] <= now and not stopping:
                release, sid = heapq.heappop(due)
                batch.append((sid, release))
            if batch:
                sids = np.array([sid for sid, _ in batch], np.int32)
                frames, later = [], []
                for sid, _ in batch:
                    s = live[sid]
                    frames.append(self.pool.frame(s.req.width, s.req.height, s.req.seed, s.queued))
                    s.queued += 1
                    if s.queued < s.req.frames:
                        later.append((s.start + s.queued / fps, sid))
                e.submit_frames(sids, frames, wait=False)
                e.step()
                in_step[step_no] = batch
                steps += 1
                for item in later:
                    heapq.heappush(due, item)
                if prev is not None:
                    e.wait_previous()      # the step before this one
                    read_step(prev)
                prev, step_no = step_no, step_no + 1
                continue
            if prev is not None:
                e.sync()
                read_step(prev)
                prev = None
            if stopping:
                for sid in list(live):
                    close(sid)
                break
            if not arrivals and not waiting and not live:
                break
            # nothing due: sleep until the next release or arrival
            nxt = [now + 0.002]
            if due:
                nxt.append(due[0][0])
            if arrivals:
                nxt.append(arrivals[0].arrival)
            wait = min(nxt) - (clock() - t0)
            if wait > 0:
                time.sleep(min(wait, 0.002))
            if now >= duration + 600.0:
                raise RuntimeError("serving did not drain within 600 s of the end")
        el = clock() - t0 if drain else min(clock() - t0, duration)
        return ServeStats(el, st["pictures"], st["mbs"], steps, admitted, len(refused), max_live, st["max_bytes"],
                          np.asarray(lat, np.float64), np.asarray(rel, np.float64))

    def _bytes(self, r: Request) -> int:
        from .engine import session_config_bytes
        return session_config_bytes(r.width, r.height, bitstream=1, quant=r.quant)
