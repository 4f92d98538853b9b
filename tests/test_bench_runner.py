"""The bench's stream bookkeeping on the CPU (no GPU, a stand-in engine):
every stream plays its clip forwards and backwards, a stream that reaches
its length is replaced by a new session and its old one is closed only once
the step holding its last picture has been read, and the device-picture
batch names each stream's current picture."""
import ctypes

import numpy as np

import bench
from h261enc_cuda_b200 import workloads


class _Engine:
    def __init__(self):
        self.next_sid, self.closed, self.device_batch = 0, [], None

    def open(self, *args, **kw):
        self.next_sid += 1
        return self.next_sid

    def close(self, sid):
        self.closed.append(sid)

    def submit_device_batch(self, sids, y, cb, cr):
        self.device_batch = (np.array(sids), np.array(y), np.array(cb), np.array(cr))

    def submit_batch_ptrs(self, n, sids_ptr, y_ptr, cb_ptr, cr_ptr, quants_ptr=0, wait=True):
        arr = lambda p, t: np.ctypeslib.as_array((t * n).from_address(p)).copy()
        self.host_batch = (arr(sids_ptr, ctypes.c_int32), arr(y_ptr, ctypes.c_uint64), arr(cb_ptr, ctypes.c_uint64),
                           arr(cr_ptr, ctypes.c_uint64))


class _Stream:
    def __init__(self, length, w=176, h=144):
        self.width, self.height, self.quant, self.length = w, h, 8, length


def _pools(n, clip_len):
    # device plane addresses: stream k, picture i -> 1000 k + 10 i (+1 Cb, +2 Cr)
    return [(None, np.zeros((clip_len, 38016), np.uint8),
             [(1000 * k + 10 * i, 1000 * k + 10 * i + 1, 1000 * k + 10 * i + 2) for i in range(clip_len)])
            for k in range(n)]


def test_runner_advances_restarts_and_retires():
    lengths = [30, 47, 100]
    streams = [_Stream(n) for n in lengths]
    e = _Engine()
    run = bench.Runner(e, streams, _pools(len(streams), bench.CLIP_LEN))
    first_sids = list(run.sids)
    pos = [0] * len(streams)
    for step in range(240):
        run.queue_device()
        sids, y, cb, cr = e.device_batch
        for k, s in enumerate(streams):
            if pos[k] >= s.length:
                pos[k] = 0
            i = workloads.clip_index(pos[k], bench.CLIP_LEN)
            pos[k] += 1
            assert y[k] == 1000 * k + 10 * i and cb[k] == y[k] + 1 and cr[k] == y[k] + 2, (step, k)
        assert list(sids) == list(run.sids)
        # read two steps behind, as the end-to-end loop does
        if step >= 2:
            last_of = dict(run.ending)
            before = len(e.closed)
            run.retire(step - 2)
            for sid in e.closed[before:]:
                assert last_of[sid] <= step - 2, f"session {sid} closed before its last step was read"
    # every replaced session was closed once its last step had been read,
    # and never before
    ended = sum((240 - 1) // n for n in lengths)   # restarts at steps n, 2n, ... below 240
    assert len(e.closed) + len(run.ending) == ended
    assert first_sids[0] in e.closed
    for sid, last in run.ending:
        assert last > 240 - 3 and sid not in e.closed


def test_runner_host_batch_addresses():
    """The host-picture batch, written in place into arrays whose addresses
    the submission takes: each stream's current clip picture and its planes,
    across restarts."""
    lengths = [30, 47, 100]
    streams = [_Stream(n) for n in lengths]
    e = _Engine()
    pools = _pools(len(streams), bench.CLIP_LEN)
    run = bench.Runner(e, streams, pools)
    pos = [0] * len(streams)
    for step in range(240):
        run.queue_host(wait=False)
        sids, y, cb, cr = e.host_batch
        assert list(sids) == list(run.sids)
        for k, s in enumerate(streams):
            if pos[k] >= s.length:
                pos[k] = 0
            i = workloads.clip_index(pos[k], bench.CLIP_LEN)
            pos[k] += 1
            base = pools[k][1].ctypes.data + i * pools[k][1].shape[1]
            assert y[k] == base and cb[k] == base + 176 * 144 and cr[k] == base + 176 * 144 * 5 // 4, (step, k)
