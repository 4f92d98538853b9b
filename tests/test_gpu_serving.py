"""Serving on the GPU: sessions arriving over time, admitted under an HBM
budget and batched continuously; every kept session's bitstream must be the
one it produces alone (the oracle's frame loop on the same pictures)."""
import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import serving, synth
from h261enc_cuda_b200.engine import Engine, session_config_bytes

pytestmark = pytest.mark.gpu


def test_served_sessions_equal_their_alone_encodes(gpu):
    reqs = serving.poisson_requests(30, 1.5, seed=11, frames=(4, 14))
    assert len(reqs) >= 20
    keep = [r.rid for r in reqs[::4]]
    # room for about six CIF sessions: later arrivals wait for earlier ones
    budget = 6 * session_config_bytes(352, 288, bitstream=1)
    pool = serving.ClipPool(clips_per_size=3, length=10)
    with Engine(max_sessions=64, levels_to_host=0, hbm_budget_bytes=budget, warps_per_cta=4) as e:
        srv = serving.Server(e, pool, fps=30.0, keep_bits_for=keep)
        st = srv.run(reqs, duration=1.5, drain=True)
    assert st.admitted == len(reqs) and st.pictures == sum(r.frames for r in reqs)
    assert st.max_session_bytes <= budget
    assert st.refused_at_least_once > 0
    for r in reqs:
        if r.rid not in keep:
            continue
        frames = np.stack([pool.frame(r.width, r.height, r.seed, i) for i in range(r.frames)])
        want = O.encode_stream(frames, r.width, r.height, quant=r.quant)[0]
        got = srv.bits[r.rid]
        assert len(got) == r.frames
        assert b"".join(got) == want, f"request {r.rid}"
    summ = st.summary()
    assert summ["latency_ms"]["p50"] is not None and summ["latency_ms"]["p99"] >= summ["latency_ms"]["p50"]


def test_served_sessions_survive_a_full_host_arena(gpu):
    """With a host bitstream arena far too small for a step, pictures that do
    not fit are read from the device, and every stream is still its alone
    encode."""
    reqs = serving.poisson_requests(40, 1.0, seed=12, frames=(3, 8))
    keep = [r.rid for r in reqs]
    pool = serving.ClipPool(clips_per_size=2, length=8)
    with Engine(max_sessions=64, levels_to_host=0, bits_host_bytes=4096, warps_per_cta=4) as e:
        srv = serving.Server(e, pool, fps=30.0, keep_bits_for=keep)
        st = srv.run(reqs, duration=1.0, drain=True)
    assert st.pictures == sum(r.frames for r in reqs)
    for r in reqs:
        frames = np.stack([pool.frame(r.width, r.height, r.seed, i) for i in range(r.frames)])
        want = O.encode_stream(frames, r.width, r.height, quant=r.quant)[0]
        assert b"".join(srv.bits[r.rid]) == want, f"request {r.rid}"


def test_reserved_blocks_serve_later_opens(gpu):
    """Blocks reserved up front are what later sessions get: opening them
    allocates no more device memory."""
    with Engine(max_sessions=64, levels_to_host=0, warps_per_cta=4) as e:
        e.reserve(176, 144, 12, bitstream=1)
        e.reserve(352, 288, 5, bitstream=1)
        held = e.stats()[2]
        assert held >= 12 * session_config_bytes(176, 144, bitstream=1) + 5 * session_config_bytes(352, 288,
                                                                                                  bitstream=1)
        sids = [e.open(176, 144, 8, bitstream=1) for _ in range(12)] + \
               [e.open(352, 288, 8, bitstream=1) for _ in range(5)]
        assert e.stats()[2] == held
        fr = synth.clip(0, 176, 144, 3, 1)[0]
        e.submit_frame(sids[0], fr)
        e.step()
        e.sync()
        assert e.result(sids[0]).bits
