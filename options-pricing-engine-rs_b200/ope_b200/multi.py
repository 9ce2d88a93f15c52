"""Multi-GPU plumbing for the pricing path: replicas / weak scaling.

Contracts and surfaces are independent (no exchange step exists on the
path), so N GPUs run N independent shards: rank r prices its own batch
(workload seed + r) with no collective on the data path.  The only
collectives are outside the timed work: a barrier before and after, and one
MAX all-reduce of the per-rank elapsed time (the job is as slow as its
slowest rank).  Works with any torch.distributed backend (NCCL on GPUs, gloo
on CPU for tests).
"""
from __future__ import annotations

import datetime
import os


def rank_info() -> tuple[int, int, int]:
    """(rank, local_rank, world_size) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def shard_seed(base_seed: int, rank: int) -> int:
    """Seed of rank `rank`'s shard: every rank prices a different batch of the same shape."""
    return base_seed + rank


def init(backend: str, timeout_s: float = 300.0):
    """Initialise the process group when WORLD_SIZE > 1; returns torch.distributed or None."""
    _, _, world = rank_info()
    if world <= 1:
        return None
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, x: float, device=None) -> float:
    """The largest value of x across ranks (the job's time is its slowest rank's)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(world: int, units_per_rank: int, steps: int, max_seconds: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return world * units_per_rank * steps / max_seconds
