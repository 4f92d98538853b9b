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


def test_one_rank_needs_no_process_group(monkeypatch):
    from h261enc_cuda_b200 import shard
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert shard.rank_info() == (1, 0, 0)
    assert shard.init("gloo") is None
    assert shard.max_over_ranks(3.0, None) == 3.0 and shard.sum_over_ranks(3.0, None) == 3.0
    shard.finish(None)
