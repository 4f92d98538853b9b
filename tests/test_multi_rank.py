"""The multi-GPU layout's host side with two ranks over gloo on the CPU:
every rank encodes its own sessions (disjoint streams, same workload
shape), and only the measurement crosses ranks (max of device times, sum of
throughputs).  One process per rank, as one process per GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from h261enc_cuda_b200 import shard
    dist = shard.init("gloo", timeout_s=60)
    w, r, local = shard.rank_info()
    streams = shard.rank_streams("batch64", r)
    seeds = [s.seed for s in streams]
    gathered = [None] * w
    dist.all_gather_object(gathered, seeds)
    out[r] = {
        "world": w, "local": local, "n": len(streams),
        "mb": sum(s.num_mb for s in streams),
        "disjoint": len(set(gathered[0]) & set(gathered[1])) == 0,
        "max": shard.max_over_ranks(1.5 + r, dist),
        "sum": shard.sum_over_ranks(1.5 + r, dist),
    }
    shard.finish(dist)


def test_two_ranks_shard_sessions_and_reduce_measurements():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r in (0, 1):
        assert res[r]["world"] == 2 and res[r]["local"] == r
        assert res[r]["n"] == 64 and res[r]["mb"] == 40 * 99 + 24 * 396   # weak scaling: same shape per rank
        assert res[r]["disjoint"]
        assert res[r]["max"] == 2.5 and res[r]["sum"] == 4.0


def _encode_rank_streams(rank, steps):
    """Rank `rank`'s batch64 streams encoded by the oracle (the bench's CPU
    runner) for `steps` steps: the SHA-256 of every stream's bytes."""
    import hashlib

    import bench
    from h261enc_cuda_b200 import shard, workloads
    streams = shard.rank_streams("batch64", rank)
    clips = [workloads.make_clip(s, steps) for s in streams]
    run = bench.CpuRunner(streams, clips, 4, clip_len=steps, keep=True)
    try:
        mbs = sum(run.step()[0] for _ in range(steps))
        return mbs, [hashlib.sha256(b"".join(pics)).hexdigest() for pics in run.out]
    finally:
        run.close()


def _encoding_rank(rank, world, port, steps, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from h261enc_cuda_b200 import shard
    dist = shard.init("gloo", timeout_s=60)
    _, r, _ = shard.rank_info()
    mbs, digests = _encode_rank_streams(r, steps)
    out[r] = {"digests": digests, "total_mb": shard.sum_over_ranks(float(mbs), dist)}
    shard.finish(dist)


def test_two_ranks_encode_their_own_streams():
    """Each of two gloo ranks encodes its own batch64 streams (the oracle
    standing in for the GPU): rank r's bitstreams are exactly what one
    process encoding rank r's streams alone writes, and the reduced MB count
    is the sum of both ranks' work -- the data path shards with nothing
    exchanged."""
    world, port, steps = 2, _free_port(), 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_encoding_rank, args=(world, port, steps, out), nprocs=world, join=True)
        res = dict(out)
    mb_per_rank = (40 * 99 + 24 * 396) * steps
    for r in (0, 1):
        mbs, alone = _encode_rank_streams(r, steps)
        assert mbs == mb_per_rank
        assert res[r]["digests"] == alone, f"rank {r}: bitstreams differ from its streams encoded alone"
        assert res[r]["total_mb"] == 2 * mb_per_rank
    assert not set(res[0]["digests"]) & set(res[1]["digests"])


def _leaving_rank(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from h261enc_cuda_b200 import shard
    dist = shard.init("gloo", timeout_s=5)
    if rank == 1:
        return          # leaves the job between steps, without taking its collectives
    try:
        shard.max_over_ranks(1.0, dist)
        out[rank] = "no error"
    except Exception as exc:  # the lost peer surfaces as an error, not a hang
        out[rank] = type(exc).__name__


def test_a_rank_that_leaves_ends_the_others_collective_with_an_error():
    """A rank that leaves between steps (failure made on the host, no GPU
    involved): the other rank's next measurement collective ends with an
    error within the process group's short timeout instead of waiting for
    good."""
    import time
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        t = time.monotonic()
        mp.spawn(_leaving_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res.get(0) not in (None, "no error"), res
    assert time.monotonic() - t < 60


def test_one_rank_needs_no_process_group(monkeypatch):
    from h261enc_cuda_b200 import shard
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert shard.rank_info() == (1, 0, 0)
    assert shard.init("gloo") is None
    assert shard.max_over_ranks(3.0, None) == 3.0 and shard.sum_over_ranks(3.0, None) == 3.0
    shard.finish(None)
