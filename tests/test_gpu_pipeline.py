"""The engine's pipelined use: steps issued back to back on its streams, the
host reading step k-1 while step k runs, streams ending and new sessions
taking their place without a drain, and the ways of queueing pictures (one
host copy per call, the batched copy, writing in place, the batched copy
left running until the next step, device pictures one call per session or
in one batched call).  Every picture must still be bit-exact to the
oracle."""
import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import _lib, synth
from h261enc_cuda_b200.engine import Engine

pytestmark = pytest.mark.gpu


class Instance:
    """One encode stream: a clip, its oracle output and its session."""

    def __init__(self, w, h, q, n, seed):
        self.w, self.h, self.q, self.n = w, h, q, n
        self.clip = synth.clip(2, w, h, seed, n)
        self.want = O.encode_sequence(self.clip, w, h, q)
        self.sid = None
        self.pos = 0        # pictures queued
        self.seen = 0       # results checked


def _check(e, inst, where):
    r = e.result(inst.sid)
    assert r.frame_index == inst.seen, f"{where}: frame index {r.frame_index} != {inst.seen}"
    got = r.to_abi(inst.w)
    want = inst.want["mbs"][inst.seen]
    for f in ("type", "flags", "quant", "cbp"):
        assert np.array_equal(got[f], want[f]), f"{where}: {f} differs"
    assert np.array_equal(got["mv"], want["mv"]), f"{where}: vectors differ"
    assert np.array_equal(got["tcoeff"], want["tcoeff"]), f"{where}: levels differ"
    inst.seen += 1
    return r.mbs


_DEVICE_PICTURES = []


def _queue(e, live, mode):
    sids = [i.sid for i in live]
    frames = [i.clip[i.pos] for i in live]
    if mode == 0:
        for s, f in zip(sids, frames):
            e.submit_frame(s, f)
    elif mode == 1:
        e.submit_frames(sids, frames)
    elif mode == 3:
        e.submit_frames(sids, frames, wait=False)   # copies finish inside the next step()
    elif mode in (4, 5):
        # pictures already in device memory, kept until the test ends
        import torch
        dev = [torch.from_numpy(np.ascontiguousarray(f)).to("cuda") for f in frames]
        _DEVICE_PICTURES.extend(dev)
        planes = [(d.data_ptr(), d.data_ptr() + i.w * i.h, d.data_ptr() + i.w * i.h * 5 // 4)
                  for d, i in zip(dev, live)]
        if mode == 4:
            e.submit_device_batch(sids, *(np.array(c, np.uint64) for c in zip(*planes)))
        else:
            for s, p in zip(sids, planes):
                e.submit_device(s, *p)
    else:
        arena, offs = e.inputs(sids)
        for inst, f, o in zip(live, frames, offs):
            ny = inst.w * inst.h
            arena[o[0]:o[0] + ny] = f[:ny]
            arena[o[1]:o[1] + ny // 4] = f[ny:ny + ny // 4]
            arena[o[2]:o[2] + ny // 4] = f[ny + ny // 4:]
    for inst in live:
        inst.pos += 1


def test_pipelined_steps_with_turnover_match_oracle(gpu):
    # (width, height, QUANT, pictures, seed): several short streams per slot
    slots = [
        [(176, 144, 8, 3, 21), (176, 144, 10, 4, 22), (176, 144, 6, 5, 23)],
        [(352, 288, 12, 5, 31), (352, 288, 16, 2, 32), (352, 288, 9, 4, 33)],
        [(176, 144, 4, 2, 41), (352, 288, 20, 3, 42), (176, 144, 14, 6, 43)],
        [(176, 144, 24, 7, 51), (176, 144, 2, 3, 52)],
    ]
    todo = [[Instance(*spec) for spec in slot] for slot in slots]
    for k, q in enumerate(todo):
        for inst in q:
            inst.slot = k
    with Engine(warps_per_cta=4, max_sessions=16) as e:
        live = []
        for q in todo:
            inst = q.pop(0)
            inst.sid = e.open(inst.w, inst.h, inst.q)
            live.append(inst)
        prev, closing, step = None, [], 0
        while live or prev:
            if live:
                _queue(e, live, step % 6)
                assert e.step() == len(live)
            cur = list(live)
            # streams whose last picture is now queued make room for the next
            nxt = []
            for inst in live:
                if inst.pos == inst.n:
                    closing.append(inst)
                    if todo[inst.slot]:
                        new = todo[inst.slot].pop(0)
                        new.sid = e.open(new.w, new.h, new.q)
                        nxt.append(new)
                else:
                    nxt.append(inst)
            live = nxt
            if prev is not None:
                if cur:
                    e.wait_previous()
                else:
                    e.sync()
                recs = [_check(e, inst, f"step {step - 1} session {inst.sid}") for inst in
                        sorted(prev, key=lambda i: i.sid)]
                done, flat = e.step_records()
                assert done >= step - 1
                if done == step - 1:
                    assert np.array_equal(flat, np.concatenate(recs))
                # a stream is closed once its last picture has been read
                for inst in [i for i in closing if i.seen == i.n]:
                    e.close(inst.sid)
                    closing.remove(inst)
            prev = cur if cur else None
            step += 1
    for slot in todo:
        assert not slot
    assert not closing


def test_inputs_are_all_or_nothing(gpu):
    with Engine(warps_per_cta=4) as e:
        a = e.open(176, 144, 8)
        b = e.open(352, 288, 8)
        with pytest.raises(RuntimeError):
            e.inputs([a, a])
        with pytest.raises(RuntimeError):
            e.inputs([a, 99])
        arena, offs = e.inputs([b, a])     # nothing was left queued
        assert offs.shape == (2, 3) and offs[1, 0] >= offs[0, 2] + 352 * 288 // 4
        c = e.open(176, 144, 8)
        fr = synth.clip(0, 176, 144, 3, 1)[0]
        with pytest.raises(RuntimeError):
            e.submit_frames([c, a], [fr, fr])   # a is already queued
        e.submit_frames([c], [fr])
        assert e.step() == 3
        e.sync()


def test_device_batch_is_all_or_nothing(gpu):
    import torch
    with Engine(warps_per_cta=4) as e:
        a = e.open(176, 144, 8)
        b = e.open(176, 144, 8)
        fr = synth.clip(0, 176, 144, 3, 1)[0]
        d = torch.from_numpy(np.ascontiguousarray(fr)).to("cuda")
        y = d.data_ptr()
        cb, cr = y + 176 * 144, y + 176 * 144 * 5 // 4

        def planes(*yy):
            return [np.array(v, np.uint64) for v in (yy, [cb] * len(yy), [cr] * len(yy))]

        with pytest.raises(RuntimeError):
            e.submit_device_batch([a, a], *planes(y, y))        # a session twice
        with pytest.raises(RuntimeError):
            e.submit_device_batch([a, b], *planes(y, y + 8))    # Y not 16-byte aligned
        with pytest.raises(RuntimeError):
            e.submit_device_batch([a, 99], *planes(y, y))       # not open
        e.submit_device(b, y, cb, cr)
        with pytest.raises(RuntimeError):
            e.submit_device_batch([a, b], *planes(y, y))        # b already queued
        e.submit_device_batch([a], *planes(y))                  # nothing of the above stayed queued
        assert e.step() == 2
        e.sync()
        ra, rb = e.result(a).to_abi(176), e.result(b).to_abi(176)
        want = O.encode_sequence(fr[None], 176, 144, 8)["mbs"][0]
        for got in (ra, rb):
            for f in ("type", "flags", "quant", "cbp", "tcoeff"):
                assert np.array_equal(got[f], want[f]), f


def test_step_records_before_any_step(gpu):
    with Engine(warps_per_cta=4) as e:
        step, recs = e.step_records()
        assert step == -1 and recs.size == 0 and recs.dtype == _lib.RESULT_DTYPE


@pytest.mark.parametrize("preset", [2, 1])
def test_graph_replay_equals_direct_launches(gpu, preset):
    """Steps replayed from captured CUDA graphs produce what directly
    launched steps produce: records, bitstreams and reconstructions, with
    sessions of two sizes, one of them rate-controlled."""
    specs = [(176, 144, 8, 0), (352, 288, 12, 0), (352, 288, 10, 256000)]
    clips = [synth.clip(preset, w, h, 70 + k, 12) for k, (w, h, q, b) in enumerate(specs)]
    out = {}
    for graphs in (0, 1):
        got = []
        # every knob fixed: no tuning steps (which launch directly)
        with Engine(warps_per_cta=4, kernel_split=1, tail_items=1, staging=1, use_graphs=graphs) as e:
            sids = [e.open(w, h, q, bitstream=1, rate_control=1 if b else 0, bitrate=b) for (w, h, q, b) in specs]
            for i in range(clips[0].shape[0]):
                e.submit_frames(sids, [c[i] for c in clips])
                e.step()
                e.sync()
                for sid in sids:
                    r = e.result(sid)
                    got.append((r.mbs.tobytes(), r.bits, np.concatenate(e.recon(sid)).tobytes()))
            caps, reps = e.graph_stats()
        if graphs:
            # a signature is captured on its second step in a row per slot
            # (three slots)
            assert caps == 3 and reps >= 3
        else:
            assert (caps, reps) == (0, 0)
        out[graphs] = got
    assert out[0] == out[1]


def test_tuned_launch_shape_is_reused_by_later_engines(gpu):
    """An engine with every knob open tunes on its first mostly-inter steps
    (27 of them; or inherits an earlier engine's plan); a later engine on
    the device inherits the plan without trying anything."""
    fr = synth.clip(0, 176, 144, 5, 8)
    with Engine() as e:
        sid = e.open(176, 144, 8)
        for i in range(32):
            e.submit_frame(sid, fr[i % 8])
            e.step()
            e.sync()
        w, c, src = e.launch_shape()
        plan, _ = e.plan()
        assert src in (1, 2) and 1 <= w <= 8 and plan["tuning"] == 0
    with Engine() as e2:
        assert e2.launch_shape() == (w, c, 2)
        assert e2.plan()[0] == dict(plan, source=2)


def test_three_steps_in_flight_match_oracle(gpu):
    """The host issues step k and only then reads step k-2 (steps k-1 and k
    still running): every session's records and bitstream are the oracle's."""
    specs = [(176, 144, 8, 81), (352, 288, 12, 82), (176, 144, 20, 83)]
    n = 8
    insts = [Instance(w, h, q, n, seed) for (w, h, q, seed) in specs]
    bits = [b"" for _ in insts]
    with Engine(warps_per_cta=4, levels_to_host=1) as e:
        for inst in insts:
            inst.sid = e.open(inst.w, inst.h, inst.q, bitstream=1)
        def read(k):   # a fresh engine numbers its steps from 0
            e.wait_step(k)
            for j, inst in enumerate(insts):
                _check(e, inst, f"step {k} session {inst.sid}")
                bits[j] += e.result(inst.sid, copy=False).bits

        for k in range(n):
            e.submit_frames([i.sid for i in insts], [i.clip[k] for i in insts])
            e.step()
            if k >= 2:
                read(k - 2)
        read(n - 2)
        read(n - 1)
    for j, inst in enumerate(insts):
        assert bits[j] == O.encode_stream(inst.clip, inst.w, inst.h, quant=inst.q)[0], f"session {j}"


def test_sync_waits_for_every_step_in_flight(gpu):
    """Steps complete out of order: step k waits only for step k-1's encode
    kernel, not for k-1's bitstream kernels and record download on its own
    stream.  Step 0 holds 24 CIF sessions with bitstreams, step 1 only a
    QCIF session; sync() must still leave step 0's results complete (every
    CIF session's records and bytes equal the oracle's first picture)."""
    n_cif = 24
    clips = [synth.clip(2, 352, 288, 900 + k, 1) for k in range(n_cif)]
    small = synth.clip(2, 176, 144, 950, 2)
    with Engine(max_sessions=64, levels_to_host=1) as e:
        big = [e.open(352, 288, 8, bitstream=1) for _ in range(n_cif)]
        sid = e.open(176, 144, 8, bitstream=1)
        e.submit_frames(big + [sid], [c[0] for c in clips] + [small[0]])
        e.step()
        e.submit_frame(sid, small[1])
        e.step()
        e.sync()
        for k, b in enumerate(big):
            want_bits, _, _, _ = O.encode_stream(clips[k], 352, 288, quant=8)
            want = O.encode_sequence(clips[k], 352, 288, 8)
            r = e.result(b)
            assert r.frame_index == 0 and r.bits_status == 0
            assert r.bits == want_bits, f"session {k}: bytes differ"
            got = r.to_abi(352)
            assert np.array_equal(got["tcoeff"], want["mbs"][0]["tcoeff"]), f"session {k}: levels differ"
            assert np.array_equal(got["type"], want["mbs"][0]["type"]), f"session {k}: types differ"


def test_batch_by_address_matches_oracle_stream(gpu):
    """Engine.submit_batch_ptrs: the caller's own session and plane-address
    arrays, rewritten in place every step and handed over by address, the
    copies left running until the next step; bitstreams, records and
    reconstructions equal the oracle's."""
    specs = [(176, 144, 8, 91), (352, 288, 12, 92), (176, 144, 20, 93)]
    n = 5
    clips = [synth.clip(2, w, h, seed, n) for (w, h, q, seed) in specs]
    ref = [O.encode_stream(c, w, h, quant=q) for c, (w, h, q, _) in zip(clips, specs)]
    want, want_rec = [r[0] for r in ref], [r[3] for r in ref]
    got = [b"" for _ in specs]
    k = len(specs)
    with Engine(warps_per_cta=4, levels_to_host=0) as e:
        sids = np.array([e.open(w, h, q, bitstream=1) for (w, h, q, _) in specs], np.int32)
        y, cb, cr = (np.zeros(k, np.uint64) for _ in range(3))
        for i in range(n):
            for j, (w, h, q, _) in enumerate(specs):
                y[j] = clips[j][i].ctypes.data
                cb[j] = y[j] + w * h
                cr[j] = cb[j] + w * h // 4
            e.submit_batch_ptrs(k, sids.ctypes.data, y.ctypes.data, cb.ctypes.data, cr.ctypes.data, wait=False)
            e.step()
            e.sync()
            for j, sid in enumerate(sids):
                got[j] += e.result(int(sid)).bits
                assert np.array_equal(np.concatenate(e.recon(int(sid))), want_rec[j][i]), (j, i)
    for j in range(k):
        assert got[j] == want[j], f"session {j}"
