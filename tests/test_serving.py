"""The serving loop's bookkeeping on the CPU, with a stand-in engine that
keeps the library's contract (steps complete in order; a step's pictures
are readable once it has completed; an HBM budget refuses sessions)."""
import numpy as np

from h261enc_cuda_b200 import serving
from h261enc_cuda_b200._lib import ERR_BUDGET, H261Error, PICTURE_DTYPE


class FakeEngine:
    def __init__(self, budget_sessions):
        self.budget = budget_sessions
        self.open_ = {}
        self.next_id = 0
        self.queued = []
        self.steps = []            # per step: (session id, picture index)
        self.done = -1
        self.closed = []

    def open(self, w, h, q, bitstream=0):
        if len(self.open_) >= self.budget:
            raise H261Error("budget", ERR_BUDGET)
        sid = self.next_id
        self.next_id += 1
        self.open_[sid] = 0
        return sid

    def close(self, sid):
        del self.open_[sid]
        self.closed.append(sid)

    def submit_frames(self, sids, frames, wait=True):
        for s in sids:
            assert int(s) in self.open_
            self.queued.append((int(s), self.open_[int(s)]))
            self.open_[int(s)] += 1

    def step(self):
        self.steps.append(self.queued)
        self.queued = []

    def wait_previous(self):
        self.done = len(self.steps) - 2

    def sync(self):
        self.done = len(self.steps) - 1

    def step_pictures(self, cap):
        out = np.zeros(len(self.steps[self.done]), PICTURE_DTYPE)
        for i, (sid, idx) in enumerate(self.steps[self.done]):
            out[i]["session_id"] = sid
            out[i]["frame_index"] = idx
            out[i]["bytes"] = 100
        return out, np.empty(0, np.uint8)


class TinyPool:
    def frame(self, w, h, seed, index):
        return np.zeros(w * h * 3 // 2, np.uint8)


def test_poisson_requests_shape():
    r = serving.poisson_requests(200, 10.0, seed=3)
    assert 1600 < len(r) < 2400
    arr = np.array([x.arrival for x in r])
    assert (np.diff(arr) > 0).all() and arr.max() < 10.0
    cif = np.mean([x.width == 352 for x in r])
    assert 0.25 < cif < 0.35
    assert all(30 <= x.frames <= 600 and 4 <= x.quant <= 24 for x in r)


def test_every_picture_once_in_order_and_budget_admission(monkeypatch):
    reqs = serving.poisson_requests(400, 0.05, seed=5, frames=(3, 9))
    eng = FakeEngine(budget_sessions=4)
    srv = serving.Server(eng, TinyPool(), fps=1000.0)
    monkeypatch.setattr(srv, "_bytes", lambda r: 1)
    st = srv.run(reqs, duration=0.05, drain=True)
    # every request served, each picture once and in order, never more than
    # the budget's sessions open at a time
    assert st.admitted == len(reqs)
    assert st.pictures == sum(r.frames for r in reqs)
    assert st.max_concurrent <= 4
    per = {}
    for s in eng.steps:
        sids = [sid for sid, _ in s]
        assert len(sids) == len(set(sids)), "a session twice in one step"
        for sid, idx in s:
            assert idx == per.get(sid, -1) + 1
            per[sid] = idx
    assert sorted(eng.closed) == list(range(len(reqs)))
    assert st.latencies_ms.size == st.pictures and (st.latencies_ms >= 0).all()
    if len(reqs) > 4:
        assert st.refused_at_least_once > 0


def test_capacity_plan_follows_littles_law():
    # 200 sessions/s, 315 pictures at 30 per second: 2,100 open at once
    assert serving.expected_concurrency(200.0, 315.0, 30.0, 1.0, margin=1.0) == 2100
    qcif = serving.expected_concurrency(200.0, 315.0, 30.0, 0.7)
    cif = serving.expected_concurrency(200.0, 315.0, 30.0, 0.3)
    assert qcif + cif >= 2100 * 1.25

    class Recorder:
        def __init__(self):
            self.calls = []

        def reserve(self, w, h, n, bitstream=0):
            self.calls.append(("blocks", w, h, n, bitstream))

        def reserve_step(self, w, h, n):
            self.calls.append(("step", w, h, n))

    rec = Recorder()
    serving.Server(rec, None).plan({(176, 144): qcif, (352, 288): cif}, burst=0.5)
    assert rec.calls == [("blocks", 176, 144, qcif, 1), ("step", 176, 144, -(-qcif // 2)),
                         ("blocks", 352, 288, cif, 1), ("step", 352, 288, -(-cif // 2))]
