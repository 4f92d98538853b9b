"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle.

Wraps oracle/_build/liboracle.so (the C restatement of the reference's
device path, h261_oracle.c) and the reference-built helpers in oracle/_ref/
(the reference's own bitstream writers, and the frame-loop drivers).  Only
tests, the smoke check and the benchmark's CPU-baseline leg import this; the
encoder library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_float, c_int8, c_int32, c_uint8, c_uint32, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
WRITER_SO = os.path.join(REF_DIR, "libh261ref_writer.so")
DRIVERS = {
    "oracle": os.path.join(REF_DIR, "h261_drive_oracle"),
    "refgpu": os.path.join(REF_DIR, "h261_drive_refgpu"),
    "refgpu_nofmad": os.path.join(REF_DIR, "h261_drive_refgpu_nofmad"),
    "ours": os.path.join(REF_DIR, "h261_drive_ours"),
}

ME_MB_DTYPE = np.dtype([("intra", "<i4"), ("zero", "<i4"), ("cost", "<i4"), ("fcost", "<i4"),
                        ("mvx", "i1"), ("mvy", "i1"), ("pad", "<i2")])
MD_DTYPE = np.dtype([("cost", "<i4"), ("qadj", "<i4"), ("type", "<i4"), ("flags", "<i4"),
                     ("mvx", "<i4"), ("mvy", "<i4")])
MB_DTYPE = np.dtype([("addr", "<i4"), ("type", "<i4"), ("flags", "<i4"), ("quant", "<i4"),
                     ("mv", "<i4", 2), ("cbp", "<i4"), ("tcoeff", "<i4", (6, 64)),
                     ("mb_x", "<i4"), ("mb_y", "<i4")])

_lib = None
_writer = None


def build() -> None:
    """Build the oracle (and, where the reference sources exist, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_fdct8x8.argtypes = [c_void_p, c_void_p, c_int32]
        L.orc_idct8x8.argtypes = [c_void_p, c_void_p, c_int32]
        L.orc_tree_reduce.argtypes = [c_int32, c_void_p, c_void_p, c_void_p]
        L.orc_satd4x4.argtypes = [c_void_p]
        L.orc_satd4x4.restype = c_int32
        L.orc_me_frame.argtypes = [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p]
        L.orc_mode_decision.argtypes = [c_void_p, c_int32, c_int32, c_void_p]
        L.orc_inv_quant.argtypes = [c_int32]
        L.orc_inv_quant.restype = c_float
        L.orc_loop_filter_hv.argtypes = [c_void_p, c_int32, c_int32, c_int32, c_void_p]
        L.orc_loop_filter_vh.argtypes = [c_void_p, c_int32, c_int32, c_int32, c_void_p]
        L.orc_mv_limits.argtypes = [c_int32, c_int32, c_void_p]
        L.orc_encode_sequence.argtypes = [c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32,
                                          c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p]
        L.orc_encode_sequence.restype = c_int32
        L.orc_write_picture.argtypes = [c_int32] * 5 + [c_void_p, c_void_p, c_int32]
        L.orc_write_picture.restype = c_int32
        L.orc_zigzag.restype = POINTER(c_uint8)
        L.orc_encode_stream.argtypes = [c_void_p] + [c_int32] * 9 + [c_void_p, ctypes.c_int64, c_void_p,
                                                                        c_void_p, c_void_p]
        L.orc_encode_stream.restype = ctypes.c_int64
        L.orc_stream_open.argtypes = [c_int32] * 8
        L.orc_stream_open.restype = c_void_p
        L.orc_stream_encode.argtypes = [c_void_p, c_void_p, c_void_p, c_int32, POINTER(c_int32), c_void_p]
        L.orc_stream_encode.restype = c_int32
        L.orc_stream_close.argtypes = [c_void_p]
        L.orc_decode_stream.argtypes = [c_void_p, ctypes.c_int64, c_int32, c_void_p, c_int32, c_void_p,
                                        POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]
        L.orc_decode_stream.restype = ctypes.c_int64
        L.orc_psnr.argtypes = [c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p]
        L.orc_rc_init.argtypes = [c_void_p, c_int32, c_int32, c_int32]
        L.orc_rc_picture_quant.argtypes = [c_void_p, c_int32, c_int32, c_int32]
        L.orc_rc_picture_quant.restype = c_int32
        L.orc_rc_update.argtypes = [c_void_p, c_int32, c_int32, c_int32]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else c_void_p(a.ctypes.data)


def fdct(block: np.ndarray, fmad: int = 1) -> np.ndarray:
    x = np.ascontiguousarray(block, np.int32).reshape(64)
    out = np.zeros(64, np.int32)
    lib().orc_fdct8x8(_p(x), _p(out), fmad)
    return out


def idct(block: np.ndarray, fmad: int = 1) -> np.ndarray:
    x = np.ascontiguousarray(block, np.int32).reshape(64)
    out = np.zeros(64, np.int32)
    lib().orc_idct8x8(_p(x), _p(out), fmad)
    return out


def tree_reduce(cost: np.ndarray, vx: np.ndarray, vy: np.ndarray):
    """Literal reference tie-break tree on a D x D grid; returns (cost, vx, vy)."""
    D = cost.shape[0]
    c = np.ascontiguousarray(cost, np.uint32).copy()
    x = np.ascontiguousarray(vx, np.int8).copy()
    y = np.ascontiguousarray(vy, np.int8).copy()
    lib().orc_tree_reduce(D, _p(c), _p(x), _p(y))
    return int(c.flat[0]), int(x.flat[0]), int(y.flat[0])


def encode_sequence(frames: np.ndarray, width: int, height: int, quant: int, intra_period: int = 0,
                    denoise: int = 5, fmad: int = 1, me_mode: int = 0):
    """Oracle encode of packed frames (n, W*H*3/2): dict of per-frame arrays."""
    n = frames.shape[0]
    nmb = (width // 16) * (height // 16)
    fr = np.ascontiguousarray(frames, np.uint8)
    recon = np.zeros_like(fr)
    mbs = np.zeros((n, nmb), MB_DTYPE)
    me = np.zeros((n, nmb), ME_MB_DTYPE)
    md = np.zeros((n, nmb), MD_DTYPE)
    rc = lib().orc_encode_sequence(_p(fr), width, height, n, quant, intra_period, denoise, fmad, me_mode,
                                   _p(recon), _p(mbs), _p(me), _p(md))
    if rc < 0:
        raise ValueError("orc_encode_sequence: bad arguments")
    return {"recon": recon, "mbs": mbs, "me": me, "md": md}


def write_picture_oracle(mbs: np.ndarray, width: int, height: int, frame_num: int, frame_type: int,
                         quant: int) -> bytes:
    """H.261 bytes of one picture from h261_macroblock_t records, written by
    the oracle's restatement of the reference writers (h261_writer.c)."""
    m = np.ascontiguousarray(mbs, MB_DTYPE)
    buf = np.zeros(400 * 1024, np.uint8)
    n = lib().orc_write_picture(width, height, frame_num, frame_type, quant, _p(m), _p(buf), buf.size)
    if n < 0:
        raise ValueError(f"orc_write_picture: status {n}")
    return buf[:n].tobytes()


def zigzag() -> np.ndarray:
    """Transmission order: raster index (row = vertical frequency) of the
    k-th coefficient sent."""
    return np.ctypeslib.as_array(lib().orc_zigzag(), shape=(64,)).copy()


def encode_stream(frames: np.ndarray, width: int, height: int, quant: int = 0, bitrate: int = 384000,
                  intra_period: int = 0, denoise: int = 5, fmad: int = 1, me_mode: int = 0):
    """The reference's frame loop with its bitstream: fixed QUANT, or CBR
    rate control when quant == 0.  Returns (bytes, per-picture byte counts,
    per-picture QUANT, reconstructions)."""
    n = frames.shape[0]
    fr = np.ascontiguousarray(frames, np.uint8)
    recon = np.zeros_like(fr)
    cap = n * 400 * 1024
    bits = np.zeros(cap, np.uint8)
    nb = np.zeros(n, np.int32)
    nq = np.zeros(n, np.int32)
    total = lib().orc_encode_stream(_p(fr), width, height, n, quant, bitrate, intra_period, denoise, fmad,
                                    me_mode, _p(bits), cap, _p(nb), _p(nq), _p(recon))
    if total < 0:
        raise ValueError(f"orc_encode_stream: status {total}")
    return bits[:total].tobytes(), nb, nq, recon


class Stream:
    """One encode stream of the oracle's frame loop, a picture at a time
    (orc_stream_*): ``encode(picture)`` returns the picture's H.261 bytes.
    The C call releases the GIL, so streams encode in parallel on threads."""

    def __init__(self, width: int, height: int, quant: int = 0, bitrate: int = 384000, intra_period: int = 0,
                 denoise: int = 5, fmad: int = 1, me_mode: int = 0):
        self._h = lib().orc_stream_open(width, height, quant, bitrate, intra_period, denoise, fmad, me_mode)
        if not self._h:
            raise ValueError(f"orc_stream_open: no stream of {width}x{height} QUANT {quant}")
        self._out = np.empty(400 * 1024, np.uint8)
        self.quant = 0

    def encode(self, picture: np.ndarray) -> bytes:
        n = self.encode_count(picture)
        return self._out[:n].tobytes()

    def encode_count(self, picture: np.ndarray) -> int:
        """Encode and return the byte count only (the bytes stay in an
        internal buffer until the next call)."""
        q = c_int32()
        n = lib().orc_stream_encode(self._h, _p(np.ascontiguousarray(picture, np.uint8)), _p(self._out),
                                    self._out.size, ctypes.byref(q), None)
        if n < 0:
            raise ValueError(f"orc_stream_encode: status {n}")
        self.quant = q.value
        return n

    def close(self) -> None:
        if self._h:
            lib().orc_stream_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def decode_stream(bits: bytes, max_frames: int = 1024, fmad: int = 1):
    """The conformance decoder: (reconstructions (n, W*H*3/2), records (n,
    nmb), width, height) of an H.261 stream of one format."""
    buf = np.frombuffer(bits, np.uint8)
    # pictures are stored back to back at their own size
    recon = np.zeros(max_frames * 352 * 288 * 3 // 2, np.uint8)
    mbs = np.zeros(max_frames * 396, MB_DTYPE)
    n, w, h = c_int32(), c_int32(), c_int32()
    used = lib().orc_decode_stream(_p(buf), buf.size, fmad, _p(recon), max_frames, _p(mbs), ctypes.byref(n),
                                   ctypes.byref(w), ctypes.byref(h))
    if used < 0:
        raise ValueError(f"orc_decode_stream: picture {-1 - used} does not parse")
    fs, nmb, k = w.value * h.value * 3 // 2, (w.value // 16) * (h.value // 16), n.value
    return recon[:k * fs].reshape(k, fs).copy(), mbs[:k * nmb].reshape(k, nmb).copy(), w.value, h.value


def psnr(orig: np.ndarray, recon: np.ndarray, width: int, height: int):
    """((ssd_y, ssd_cb, ssd_cr), (psnr_y, psnr_cb, psnr_cr)) of one picture,
    the reference's get_frame_psnr."""
    ssd = np.zeros(3, np.uint64)
    out = np.zeros(3, np.float64)
    lib().orc_psnr(_p(np.ascontiguousarray(orig, np.uint8)), _p(np.ascontiguousarray(recon, np.uint8)), width,
                   height, _p(ssd), _p(out))
    return tuple(int(x) for x in ssd), tuple(float(x) for x in out)


class RateControl:
    """The oracle's restatement of the reference rate control."""

    def __init__(self, quant: int = 10, bitrate: int = 384000, vbv: int | None = None):
        self._s = (c_int32 * 9)()
        lib().orc_rc_init(ctypes.byref(self._s), quant, bitrate, bitrate if vbv is None else vbv)

    def picture_quant(self, frame_type: int, picture_cost: int, num_mb: int) -> int:
        return lib().orc_rc_picture_quant(ctypes.byref(self._s), frame_type, picture_cost, num_mb)

    def update(self, frame_type: int, quant: int, nbytes: int) -> None:
        lib().orc_rc_update(ctypes.byref(self._s), frame_type, quant, nbytes)

    def state(self):
        return list(self._s)


def me_frame(cur_y: np.ndarray, ref_y: np.ndarray, width: int, height: int, mode: int = 0):
    nmb = (width // 16) * (height // 16)
    out = np.zeros(nmb, ME_MB_DTYPE)
    s1 = np.zeros(nmb * 2, np.int8)
    lib().orc_me_frame(_p(np.ascontiguousarray(cur_y)), _p(np.ascontiguousarray(ref_y)), width, height, mode,
                       _p(out), _p(s1))
    return out, s1.reshape(nmb, 2)


def mode_decision(me: np.ndarray, frame_type: int) -> np.ndarray:
    md = np.zeros(me.size, MD_DTYPE)
    lib().orc_mode_decision(_p(np.ascontiguousarray(me)), me.size, frame_type, _p(md))
    return md


# ---- the reference's own bitstream writers (built from its sources) -------

def have_reference_builds() -> bool:
    return os.path.exists(WRITER_SO) and os.path.exists(DRIVERS["oracle"])


def write_picture(mbs: np.ndarray, width: int, height: int, frame_num: int, frame_type: int,
                  quant: int) -> bytes:
    """H.261 bytes of one picture from h261_macroblock_t records, written by
    the reference's h261_picture.c / h261_gob.c / h261_macroblock.c."""
    global _writer
    if _writer is None:
        _writer = ctypes.CDLL(WRITER_SO)
        _writer.ref_write_picture.argtypes = [c_int32] * 5 + [c_void_p, c_void_p, c_int32]
        _writer.ref_write_picture.restype = c_int32
    m = np.ascontiguousarray(mbs, MB_DTYPE).copy()
    buf = np.zeros(1 << 20, np.uint8)
    n = _writer.ref_write_picture(width, height, frame_num, frame_type, quant, _p(m), _p(buf), buf.size)
    if n < 0:
        raise ValueError("bitstream buffer too small")
    return buf[:n].tobytes()


def run_driver(kind: str, yuv_path: str, width: int, height: int, frames: int, out_dir: str,
               quant: int = 0, bitrate: int = 384000, intra: int = 0, denoise: int = 5, env=None,
               timeout: float = 600.0):
    """Run one frame-loop driver; returns paths of (bits, recon, dump)."""
    exe = DRIVERS[kind]
    bits = os.path.join(out_dir, f"{kind}.h261")
    recon = os.path.join(out_dir, f"{kind}_recon.yuv")
    dump = os.path.join(out_dir, f"{kind}.dump")
    args = [exe, f"in={yuv_path}", f"w={width}", f"h={height}", f"frames={frames}", f"bits={bits}",
            f"recon={recon}", f"dump={dump}", f"intra={intra}", f"denoise={denoise}"]
    args.append(f"quant={quant}" if quant > 0 else f"bitrate={bitrate}")
    e = dict(os.environ)
    if env:
        e.update(env)
    subprocess.run(args, check=True, stdout=subprocess.DEVNULL, env=e, timeout=timeout)
    return bits, recon, dump


def read_dump(path: str):
    """Frames of a driver dump: list of dicts (header, me, md, mbs)."""
    b = open(path, "rb").read()
    o, out = 0, []
    while o < len(b):
        if b[o:o + 8] != b"H261FRM1":
            raise ValueError(f"bad dump record at {o}")
        o += 8
        f, t, q, n, ln = np.frombuffer(b, "<i4", 5, o)
        o += 20
        me = np.frombuffer(b, ME_MB_DTYPE, n, o)
        o += n * 20
        md = np.frombuffer(b, MD_DTYPE, n, o)
        o += n * 24
        mbs = np.frombuffer(b, MB_DTYPE, n, o)
        o += n * 1572
        out.append({"frame": int(f), "type": int(t), "quant": int(q), "num_mb": int(n), "bytes": int(ln),
                    "me": me, "md": md, "mbs": mbs})
    return out
