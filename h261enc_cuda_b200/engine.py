"""Batched encode engine (include/h261b.h) from Python.

One ``Engine`` owns a CUDA stream, a device pool and the double-buffered
upload / result arenas.  Sessions are independent encode streams; each
``step()`` encodes the queued picture of every session in one launch.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check


@dataclass
class FrameResult:
    frame_index: int
    frame_type: int
    quant: int
    mbs: np.ndarray        # RESULT_DTYPE[num_mb]
    levels: np.ndarray     # int8 [num_mb, 6, 64], per block column-major (u * 8 + v); None if not copied
    bits: bytes = None     # the picture's H.261 bytes (sessions opened with bitstream=1)
    bits_status: int = 0
    psnr: tuple = None     # (Y, Cb, Cr) dB, sessions opened with psnr=1
    ssd: tuple = None      # the squared errors they come from

    def to_abi(self, width: int) -> np.ndarray:
        """The reference's h261_macroblock_t array for this picture."""
        out = np.zeros(self.mbs.size, _lib.MB_DTYPE)
        out["type"] = self.mbs["type"]
        out["flags"] = self.mbs["flags"]
        out["quant"] = self.mbs["quant"]
        out["mv"][:, 0] = self.mbs["mvx"]
        out["mv"][:, 1] = self.mbs["mvy"]
        out["cbp"] = self.mbs["cbp"].astype(np.uint8)
        n = self.mbs.size
        raster = self.levels.reshape(n, 6, 8, 8).transpose(0, 1, 3, 2).reshape(n, 6, 64)
        tc = raster.astype(np.int32)
        intra = self.mbs["type"] == _lib.MB_TYPE_INTRA
        tc[intra, :, 0] = raster[intra, :, 0].view(np.uint8)
        out["tcoeff"] = tc
        mbw = width // 16
        idx = np.arange(self.mbs.size)
        out["mb_x"] = (idx % mbw) * 16
        out["mb_y"] = (idx // mbw) * 16
        return out


class Engine:
    def __init__(self, device: int = 0, max_sessions: int = 4096, hbm_budget_bytes: int = 0,
                 me_mode: int = 0, fmad: int = 1, warps_per_cta: int = 0, max_ctas: int = 0,
                 copy_threads: int = 0, levels_to_host: int = 1, bits_host_bytes: int = 0,
                 use_graphs: int = 1, kernel_split: int = 0, tail_items: int = 0, staging: int = 0):
        lib = _lib.core()
        cfg = _lib.EngineConfig()
        lib.h261b_engine_config_default(ctypes.byref(cfg))
        cfg.device, cfg.max_sessions, cfg.hbm_budget_bytes = device, max_sessions, hbm_budget_bytes
        cfg.me_mode, cfg.fmad, cfg.warps_per_cta, cfg.max_ctas = me_mode, fmad, warps_per_cta, max_ctas
        cfg.copy_threads = copy_threads
        cfg.levels_to_host, cfg.bits_host_bytes = levels_to_host, bits_host_bytes
        cfg.use_graphs = use_graphs
        cfg.kernel_split, cfg.tail_items, cfg.staging = kernel_split, tail_items, staging
        h = ctypes.c_void_p()
        check(lib.h261b_engine_create(ctypes.byref(cfg), ctypes.byref(h)), "h261b_engine_create")
        self._h = h
        self._dims = {}

    # -- sessions
    def open(self, width: int, height: int, quant: int, intra_period: int = 0, denoise: int = 5,
             bitstream: int = 0, rate_control: int = 0, bitrate: int = 0, psnr: int = 0) -> int:
        """A new encode session.  rate_control=1: the reference's CBR rate
        control at `bitrate` bit/s on the device, starting at `quant`
        (needs bitstream=1).  psnr=1: each result carries the picture's
        PSNR."""
        c = _lib.SessionConfig(width, height, quant, intra_period, denoise, bitstream, rate_control, bitrate, psnr)
        sid = ctypes.c_int32()
        check(_lib.core().h261b_session_open(self._h, ctypes.byref(c), ctypes.byref(sid)), "h261b_session_open")
        self._dims[sid.value] = (width, height)
        return sid.value

    def reserve(self, width: int, height: int, count: int, bitstream: int = 0, rate_control: int = 0,
                bitrate: int = 0) -> None:
        """Allocate the device blocks of ``count`` sessions of this shape now,
        so that opening them later allocates nothing."""
        c = _lib.SessionConfig(width, height, 8, 0, 5, bitstream, rate_control, bitrate, 0)
        check(_lib.core().h261b_engine_reserve(self._h, ctypes.byref(c), count), "h261b_engine_reserve")

    def reserve_step(self, width: int, height: int, pictures: int) -> None:
        """Size the step arenas for ``pictures`` more pictures of this size
        in one step, so that steps up to that size never reallocate them."""
        c = _lib.SessionConfig(width, height, 8, 0, 5, 0, 0, 0, 0)
        check(_lib.core().h261b_engine_reserve_step(self._h, ctypes.byref(c), pictures), "h261b_engine_reserve_step")

    def close(self, sid: int) -> None:
        check(_lib.core().h261b_session_close(self._h, sid), "h261b_session_close")
        self._dims.pop(sid, None)

    def submit(self, sid: int, y: np.ndarray, cb: np.ndarray, cr: np.ndarray, quant: int = 0) -> None:
        check(_lib.core().h261b_session_submit(self._h, sid, _lib.ptr(y), _lib.ptr(cb), _lib.ptr(cr), quant),
              "h261b_session_submit")

    def submit_device(self, sid: int, y_ptr: int, cb_ptr: int, cr_ptr: int, quant: int = 0) -> None:
        """Queue a picture already in device memory (raw device pointers)."""
        check(_lib.core().h261b_session_submit_device(self._h, sid, ctypes.c_void_p(y_ptr), ctypes.c_void_p(cb_ptr),
                                                      ctypes.c_void_p(cr_ptr), quant), "h261b_session_submit_device")

    def input(self, sid: int, quant: int = 0):
        """Queue the session's next picture in place: returns writable numpy
        views (y, cb, cr) of the pinned staging arena; fill them before the
        next ``step()``."""
        w, h = self._dims[sid]
        py, pcb, pcr = (ctypes.POINTER(ctypes.c_uint8)() for _ in range(3))
        check(_lib.core().h261b_session_input(self._h, sid, quant, ctypes.byref(py), ctypes.byref(pcb),
                                              ctypes.byref(pcr)), "h261b_session_input")
        ny = w * h
        return (np.ctypeslib.as_array(py, shape=(ny,)), np.ctypeslib.as_array(pcb, shape=(ny // 4,)),
                np.ctypeslib.as_array(pcr, shape=(ny // 4,)))

    def inputs(self, sids, quants=None):
        """Queue the next picture of many sessions in one call: returns the
        pinned staging arena as a writable uint8 array and an int64 array
        (n, 3) of the Y, Cb, Cr plane offsets of each session in it."""
        sids = np.ascontiguousarray(sids, np.int32)
        n = sids.size
        q = None if quants is None else np.ascontiguousarray(quants, np.int32)
        offs = np.empty((n, 3), np.int64)
        base = ctypes.c_void_p()
        check(_lib.core().h261b_engine_inputs(self._h, n, sids.ctypes.data, None if q is None else q.ctypes.data,
                                              ctypes.byref(base), offs.ctypes.data), "h261b_engine_inputs")
        if n == 0:
            return np.empty(0, np.uint8), offs
        w, h = self._dims[int(sids[int(np.argmax(offs[:, 0]))])]
        size = int(offs[:, 0].max()) + w * h * 3 // 2 + 512
        arena = np.ctypeslib.as_array((ctypes.c_uint8 * size).from_address(base.value))
        return arena, offs

    def submit_device_batch(self, sids, y_ptrs, cb_ptrs, cr_ptrs, quants=None) -> None:
        """``submit_device`` for every session of ``sids`` in one call: device
        plane addresses as uint64 arrays; all or nothing."""
        sids = np.ascontiguousarray(sids, np.int32)
        ptrs = [np.ascontiguousarray(a, np.uint64) for a in (y_ptrs, cb_ptrs, cr_ptrs)]
        q = None if quants is None else np.ascontiguousarray(quants, np.int32)
        check(_lib.core().h261b_engine_submit_device_batch(self._h, sids.size, sids.ctypes.data, ptrs[0].ctypes.data,
                                                           ptrs[1].ctypes.data, ptrs[2].ctypes.data,
                                                           None if q is None else q.ctypes.data),
              "h261b_engine_submit_device_batch")

    def submit_batch(self, sids, y_ptrs, cb_ptrs, cr_ptrs, quants=None, wait: bool = True) -> None:
        """Queue one host picture for each of ``sids``: plane addresses as
        uint64 arrays (packed planes, e.g. ``frame.ctypes.data`` and the
        offsets of Cb and Cr in it).  The engine's copy threads move the
        pictures into the staging arena; with ``wait=False`` the call
        returns once they have started and the next ``step()`` waits for
        them (the source memory must stay unchanged until then)."""
        sids = np.ascontiguousarray(sids, np.int32)
        ptrs = [np.ascontiguousarray(a, np.uint64) for a in (y_ptrs, cb_ptrs, cr_ptrs)]
        q = None if quants is None else np.ascontiguousarray(quants, np.int32)
        fn = _lib.core().h261b_engine_submit_batch if wait else _lib.core().h261b_engine_submit_batch_async
        check(fn(self._h, sids.size, sids.ctypes.data, ptrs[0].ctypes.data, ptrs[1].ctypes.data,
                 ptrs[2].ctypes.data, None if q is None else q.ctypes.data), "h261b_engine_submit_batch")

    def submit_batch_ptrs(self, n: int, sids_ptr: int, y_ptr: int, cb_ptr: int, cr_ptr: int,
                          quants_ptr: int = 0, wait: bool = True) -> None:
        """``submit_batch`` with the addresses of the caller's own arrays
        (n int32 session ids, n uint64 plane addresses each, optionally n
        int32 QUANTs): no conversion on the per-step path, for a caller that
        keeps those arrays and rewrites them in place every step."""
        fn = _lib.core().h261b_engine_submit_batch if wait else _lib.core().h261b_engine_submit_batch_async
        check(fn(self._h, n, sids_ptr, y_ptr, cb_ptr, cr_ptr, quants_ptr or None), "h261b_engine_submit_batch")

    def submit_frames(self, sids, frames, quants=None, wait: bool = True) -> None:
        """``submit_batch`` for packed frames (uint8 arrays of W*H*3/2)."""
        y = np.array([f.ctypes.data for f in frames], np.uint64)
        ny = np.array([self._dims[int(s)][0] * self._dims[int(s)][1] for s in sids], np.uint64)
        self.submit_batch(sids, y, y + ny, y + ny + ny // 4, quants, wait=wait)

    def step_records(self):
        """(step number, MB records of every session that step encoded) for
        the latest completed step; a view valid until the third step after it is
        issued."""
        ptr, count, step = ctypes.c_void_p(), ctypes.c_int64(), ctypes.c_int64()
        check(_lib.core().h261b_engine_step_records(self._h, ctypes.byref(ptr), ctypes.byref(count),
                                                    ctypes.byref(step)), "h261b_engine_step_records")
        if count.value == 0:
            return step.value, np.empty(0, _lib.RESULT_DTYPE)
        buf = (ctypes.c_uint8 * (count.value * 16)).from_address(ptr.value)
        return step.value, np.ctypeslib.as_array(buf).view(_lib.RESULT_DTYPE)

    def submit_frame(self, sid: int, frame: np.ndarray, quant: int = 0) -> None:
        w, h = self._dims[sid]
        fs = w * h
        self.submit(sid, frame[:fs], frame[fs:fs + fs // 4], frame[fs + fs // 4:fs + fs // 2], quant)

    # -- steps
    def step(self) -> int:
        return check(_lib.core().h261b_engine_step(self._h), "h261b_engine_step")

    def sync(self) -> None:
        check(_lib.core().h261b_engine_sync(self._h), "h261b_engine_sync")

    def wait_step(self, step: int) -> None:
        """Wait for step number ``step`` (0, 1, ... in issue order), one of
        the last three issued; its results become the latest readable."""
        check(_lib.core().h261b_engine_wait_step(self._h, step), "h261b_engine_wait_step")

    def wait_previous(self) -> None:
        """Wait for the step before the last one issued."""
        check(_lib.core().h261b_engine_wait_previous(self._h), "h261b_engine_wait_previous")

    def result(self, sid: int, copy: bool = True) -> FrameResult:
        r = _lib.FrameResult()
        check(_lib.core().h261b_session_result(self._h, sid, ctypes.byref(r)), "h261b_session_result")
        n = r.num_mb
        mbs = np.ctypeslib.as_array((ctypes.c_uint8 * (n * 16)).from_address(r.mbs)).view(_lib.RESULT_DTYPE)
        lv = np.ctypeslib.as_array(r.levels, shape=(n * 384,)).reshape(n, 6, 64) if r.levels else None
        if copy:
            mbs = mbs.copy()
            lv = None if lv is None else lv.copy()
        bits = ctypes.string_at(r.bits, r.bits_bytes) if r.bits else None
        psnr = tuple(r.psnr) if any(r.ssd) or any(r.psnr) else None
        return FrameResult(r.frame_index, r.frame_type, r.quant, mbs, lv, bits, r.bits_status, psnr,
                           tuple(r.ssd) if psnr else None)

    def last_bits_ms(self) -> float:
        ms = ctypes.c_float()
        check(_lib.core().h261b_engine_last_bits_ms(self._h, ctypes.byref(ms)), "h261b_engine_last_bits_ms")
        return ms.value

    def step_pictures(self, cap: int = 4096):
        """(PICTURE_DTYPE array, host arena span as a uint8 view) of the
        latest completed step's bitstream output."""
        out = np.zeros(cap, _lib.PICTURE_DTYPE)
        n = ctypes.c_int32()
        base, used = ctypes.c_void_p(), ctypes.c_int64()
        check(_lib.core().h261b_engine_step_pictures(self._h, cap, out.ctypes.data, ctypes.byref(n),
                                                     ctypes.byref(base), ctypes.byref(used)),
              "h261b_engine_step_pictures")
        span = (np.ctypeslib.as_array((ctypes.c_uint8 * used.value).from_address(base.value))
                if used.value else np.empty(0, np.uint8))
        return out[:min(n.value, cap)], span

    def graph_stats(self):
        """(steps captured as CUDA graphs, steps that replayed one)."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        check(_lib.core().h261b_engine_graph_stats(self._h, ctypes.byref(a), ctypes.byref(b)),
              "h261b_engine_graph_stats")
        return a.value, b.value

    def launch_shape(self):
        """(warps per CTA, CTA cap, source: 0 configured, 1 tuned, 2 tuned
        earlier in this process on the same device)."""
        w, c, src = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check(_lib.core().h261b_engine_launch_shape(self._h, ctypes.byref(w), ctypes.byref(c), ctypes.byref(src)),
              "h261b_engine_launch_shape")
        return w.value, c.value, src.value

    def plan(self):
        """(the encode kernel's launch plan, [(candidate plan, encode ms)]
        the tuner measured): plans as dicts of warps_per_cta, max_ctas,
        kernel_split (1 fused, 2 search + encode), tail_items (n + 1),
        staging (1 cp.async, 2 bulk rows), source, tuning."""
        cap = 64
        log = (_lib.LaunchPlan * cap)()
        ms = (ctypes.c_float * cap)()
        cur, n = _lib.LaunchPlan(), ctypes.c_int32()
        check(_lib.core().h261b_engine_plan(self._h, ctypes.byref(cur), cap, log, ms, ctypes.byref(n)),
              "h261b_engine_plan")
        as_dict = lambda p: {f: getattr(p, f) for f, _ in _lib.LaunchPlan._fields_ if f != "reserved"}
        return as_dict(cur), [(as_dict(log[i]), ms[i]) for i in range(min(n.value, cap))]

    def step_timing(self) -> dict:
        """Device timeline of the latest completed step, in milliseconds."""
        t = _lib.StepTiming()
        check(_lib.core().h261b_engine_step_timing(self._h, ctypes.byref(t)), "h261b_engine_step_timing")
        return {"step": t.step, "upload": t.upload_ms, "wait": t.wait_ms, "encode": t.encode_ms,
                "bitstream": t.bitstream_ms, "total": t.total_ms}

    def step_bits(self):
        """(bytes, pictures) of bitstream the latest completed step wrote."""
        b, n = ctypes.c_int64(), ctypes.c_int32()
        check(_lib.core().h261b_engine_step_bits(self._h, ctypes.byref(b), ctypes.byref(n)),
              "h261b_engine_step_bits")
        return b.value, n.value

    def recon(self, sid: int):
        w, h = self._dims[sid]
        y = np.empty(w * h, np.uint8)
        cb = np.empty(w * h // 4, np.uint8)
        cr = np.empty(w * h // 4, np.uint8)
        check(_lib.core().h261b_session_recon(self._h, sid, _lib.ptr(y), _lib.ptr(cb), _lib.ptr(cr)),
              "h261b_session_recon")
        return y, cb, cr

    def last_kernel_ms(self) -> float:
        ms = ctypes.c_float()
        check(_lib.core().h261b_engine_last_kernel_ms(self._h, ctypes.byref(ms)), "h261b_engine_last_kernel_ms")
        return ms.value

    def last_copy_bytes(self):
        """(host-to-device, device-to-host) bytes the last step copied."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        check(_lib.core().h261b_engine_last_copy_bytes(self._h, ctypes.byref(a), ctypes.byref(b)),
              "h261b_engine_last_copy_bytes")
        return a.value, b.value

    def stats(self):
        o, q, b = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        check(_lib.core().h261b_engine_stats(self._h, ctypes.byref(o), ctypes.byref(q), ctypes.byref(b)),
              "h261b_engine_stats")
        return o.value, q.value, b.value

    def destroy(self) -> None:
        if self._h:
            _lib.core().h261b_engine_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def session_config_bytes(width: int, height: int, bitstream: int = 0, rate_control: int = 0, bitrate: int = 0,
                         quant: int = 8) -> int:
    """Device bytes (the admission charge) of a session of this configuration."""
    c = _lib.SessionConfig(width, height, quant, 0, 5, bitstream, rate_control, bitrate, 0)
    return check(_lib.core().h261b_session_config_bytes(ctypes.byref(c)), "h261b_session_config_bytes")


def session_bytes(width: int, height: int) -> int:
    return int(_lib.core().h261b_session_bytes(width, height))


def sad_peak(device: int = 0) -> float:
    """Measured 4-pixel SAD throughput of the device, absolute differences/s."""
    v = ctypes.c_double()
    if _lib.core().h261b_measure_sad_peak(device, ctypes.byref(v)) != 0:
        raise _lib.H261Error("h261b_measure_sad_peak failed")
    return v.value


def debug_check_status():
    """(enabled, failures since the last call, first failing site, its
    index) of the loaded library's bounds checks: enabled only in the
    checking build (H261B_LIB=check)."""
    en, n, site, val = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
    check(_lib.core().h261b_debug_check_status(ctypes.byref(en), ctypes.byref(n), ctypes.byref(site),
                                               ctypes.byref(val)), "h261b_debug_check_status")
    return bool(en.value), n.value, site.value, val.value


def stage_timeouts() -> int:
    """Bulk-staging waits that gave up on the current device since the last
    call (h261b_stage_status; 0 in every correct run)."""
    n = ctypes.c_int64()
    check(_lib.core().h261b_stage_status(ctypes.byref(n)), "h261b_stage_status")
    return n.value
