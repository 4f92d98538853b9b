"""h261b_encode_picture_noalloc: one picture per call, no allocation.

Some callers cannot call cudaMalloc -- their device memory belongs to
another allocator or pool, or they run where an allocation is not allowed --
so this entry point takes only caller-owned device buffers and keeps its own
scratch in a fixed static device array.  Here the caller's buffers come from
torch (the test is the caller); the library call itself allocates nothing.
Its output must equal the batched engine's (the existing entry point) bit
for bit on two calls in a row: an intra picture, then an inter picture that
uses the first call's reconstruction and denoise state.
"""
import ctypes

import numpy as np
import pytest

from h261enc_cuda_b200 import _lib, synth
from h261enc_cuda_b200.engine import Engine

pytestmark = pytest.mark.gpu


class NoallocPicture(ctypes.Structure):  # h261b_noalloc_picture_t, include/h261b.h
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("frame_type", ctypes.c_int32),
                ("quant", ctypes.c_int32), ("me_mode", ctypes.c_int32), ("fmad", ctypes.c_int32),
                ("denoise", ctypes.c_int32), ("reset_state", ctypes.c_int32)] + \
               [(n, ctypes.c_void_p) for n in ("cur_y", "cur_cb", "cur_cr", "ref_y", "ref_cb", "ref_cr",
                                              "rec_y", "rec_cb", "rec_cr", "state", "mbs", "levels")]


def _lib_noalloc():
    lib = _lib.core()
    lib.h261b_encode_picture_noalloc.argtypes = [ctypes.POINTER(NoallocPicture), ctypes.c_void_p]
    lib.h261b_encode_picture_noalloc.restype = ctypes.c_int32
    return lib


class DevPicture:
    """A caller-owned device picture: Y, Cb, Cr planes on 256-byte offsets."""

    def __init__(self, torch, w, h, host=None):
        self.w, self.h = w, h
        self.ny, self.nc = w * h, w * h // 4
        self.off_cb = (self.ny + 255) // 256 * 256
        self.off_cr = self.off_cb + (self.nc + 255) // 256 * 256
        self.buf = torch.zeros(self.off_cr + (self.nc + 255) // 256 * 256, dtype=torch.uint8, device="cuda:0")
        if host is not None:
            t = torch.from_numpy(np.ascontiguousarray(host))
            self.buf[:self.ny] = t[:self.ny].cuda()
            self.buf[self.off_cb:self.off_cb + self.nc] = t[self.ny:self.ny + self.nc].cuda()
            self.buf[self.off_cr:self.off_cr + self.nc] = t[self.ny + self.nc:].cuda()

    def planes(self):
        b = self.buf.data_ptr()
        return b, b + self.off_cb, b + self.off_cr

    def host(self):
        a = self.buf.cpu().numpy()
        return np.concatenate([a[:self.ny], a[self.off_cb:self.off_cb + self.nc],
                               a[self.off_cr:self.off_cr + self.nc]])


@pytest.mark.parametrize("w,h,me_mode,fmad", [(176, 144, 0, 1), (352, 288, 1, 0)])
def test_noalloc_matches_engine_on_two_calls(gpu, w, h, me_mode, fmad):
    import torch
    lib = _lib_noalloc()
    q = 8
    nmb = (w // 16) * (h // 16)
    frames = synth.clip(0, w, h, 41, 2)

    want = []
    with Engine(warps_per_cta=4, me_mode=me_mode, fmad=fmad) as e:
        sid = e.open(w, h, q)
        for i in range(2):
            e.submit_frame(sid, frames[i])
            e.step()
            e.sync()
            r = e.result(sid)
            want.append((r.mbs.copy(), r.levels.copy(), np.concatenate(e.recon(sid))))

    cur = [DevPicture(torch, w, h, frames[i]) for i in range(2)]
    black = DevPicture(torch, w, h)
    rec = [DevPicture(torch, w, h) for _ in range(2)]
    state = torch.zeros(_lib_state_bytes(), dtype=torch.uint8, device="cuda:0")
    mbs = torch.zeros(nmb * 16, dtype=torch.uint8, device="cuda:0")
    levels = torch.zeros(nmb * 384, dtype=torch.uint8, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    for i in range(2):
        p = NoallocPicture()
        # the strength is read on the first call only (reset_state): the
        # second call's 9 must be ignored, as the engine's session keeps 5
        p.width, p.height, p.quant, p.me_mode, p.fmad = w, h, q, me_mode, fmad
        p.denoise = 5 if i == 0 else 9
        p.frame_type = 0 if i == 0 else 1
        p.reset_state = 1 if i == 0 else 0
        p.cur_y, p.cur_cb, p.cur_cr = cur[i].planes()
        p.ref_y, p.ref_cb, p.ref_cr = (black if i == 0 else rec[0]).planes()
        p.rec_y, p.rec_cb, p.rec_cr = rec[i].planes()
        p.state, p.mbs, p.levels = state.data_ptr(), mbs.data_ptr(), levels.data_ptr()
        rc = lib.h261b_encode_picture_noalloc(ctypes.byref(p), ctypes.c_void_p(stream))
        assert rc == 0, lib.h261b_last_error()
        torch.cuda.synchronize()
        got_mbs = mbs.cpu().numpy().view(_lib.RESULT_DTYPE)
        got_lv = levels.cpu().numpy().view(np.int8).reshape(nmb, 6, 64)
        assert np.array_equal(got_mbs, want[i][0]), f"call {i + 1}: macroblock results differ"
        assert np.array_equal(got_lv, want[i][1]), f"call {i + 1}: levels differ"
        assert np.array_equal(rec[i].host(), want[i][2]), f"call {i + 1}: reconstruction differs"


def _lib_state_bytes():
    return 1040  # H261B_NOALLOC_STATE_BYTES


def test_noalloc_refuses_oversize_picture(gpu):
    import torch
    lib = _lib_noalloc()
    buf = torch.zeros(1 << 16, dtype=torch.uint8, device="cuda:0")
    b = buf.data_ptr()
    p = NoallocPicture()
    p.width, p.height, p.quant, p.frame_type, p.fmad = 1040, 1040, 8, 0, 1
    for n in ("cur_y", "cur_cb", "cur_cr", "ref_y", "ref_cb", "ref_cr", "rec_y", "rec_cb", "rec_cr", "state",
              "mbs", "levels"):
        setattr(p, n, b)
    rc = lib.h261b_encode_picture_noalloc(ctypes.byref(p), None)
    assert rc == -1
    assert b"more than the 4096" in lib.h261b_last_error()
