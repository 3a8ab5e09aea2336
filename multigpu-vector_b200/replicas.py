"""Host-side logic of running independent replicas of the join, one process per GPU.

The hash-join probe shards with no exchange (probe rows are independent given
the table), so N GPUs run N replicas of the whole workload: no collective
touches the data path.  The process group only brackets the timed region
(barriers), takes the slowest replica's time (max over ranks) and checks that
every replica computed the same result.  Backend "nccl" on GPUs; "gloo" runs
the same code on CPU processes.
"""
from __future__ import annotations

import datetime
import os


def init(backend: str, timeout_s: float = 120.0):
    """Joins the process group described by the torchrun environment.

    Returns (dist, world, rank, local_rank); dist is None for a single process."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return None, 1, 0, local
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist, world, rank, local


def max_over_ranks(dist, value: float, device="cpu") -> float:
    """The largest `value` over all ranks (every rank gets it)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, units_per_replica: float, slowest_s: float) -> float:
    """Whole-job throughput: the units all replicas processed / the slowest replica's time."""
    return world * units_per_replica / slowest_s


def same_on_all_ranks(dist, result) -> bool:
    """True when every rank passes an equal `result` (any picklable value)."""
    if dist is None:
        return True
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, result)
    return all(r == out[0] for r in out)


def finish(dist) -> None:
    """Last barrier, then leave the process group."""
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
