"""Sessions sharded across GPUs.

Encode sessions are independent: a session's pictures, reconstructions and
rate-control state never leave its GPU, and no step needs another GPU's
data.  So the path scales by giving every GPU its own process, engine and
sessions (weak scaling), with no collective on the data path.  Only the
measurement crosses ranks: device times reduce by their maximum (the job
ends when its slowest rank ends) and throughputs by their sum, through
torch.distributed (NCCL between GPUs, gloo on the CPU).
"""
from __future__ import annotations

import datetime
import os
from typing import List, Tuple

from . import workloads


def rank_info() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0):
    """torch.distributed for a multi-rank job (None for one rank).  The short
    timeout makes ranks that wait for a lost peer end with an error."""
    world, _, _ = rank_info()
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def rank_streams(workload: str, rank: int) -> List[workloads.Stream]:
    """The streams rank `rank` encodes: the workload's shape with the rank's
    own seeds, so no two ranks encode the same stream."""
    return workloads.WORKLOADS[workload](rank=rank)


def _reduce(x: float, dist, device: str, op_name: str) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(x: float, dist, device: str = "cpu") -> float:
    """The largest value over all ranks (device times: the job's time)."""
    return _reduce(x, dist, device, "MAX")


def sum_over_ranks(x: float, dist, device: str = "cpu") -> float:
    """The sum over all ranks (throughputs, pictures)."""
    return _reduce(x, dist, device, "SUM")


def finish(dist) -> None:
    """Leave the job: every rank takes the same final barrier."""
    if dist is None:
        return
    dist.barrier()
    dist.destroy_process_group()
