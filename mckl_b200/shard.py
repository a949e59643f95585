"""Sharding of the batched workloads over ranks (one process per GPU).

The path partitions into independent objects, so ranks exchange no data:
rank r runs filters [r F, (r + 1) F) of one global workload (their own
parameters, observation, model and resampling keys), and RNG fills use the
rank-private counter range (i, r) of the same key.  The only collective is
the whole-job rate: particle-steps (or bytes) summed over ranks divided by
the slowest rank's device time.
"""
from __future__ import annotations


def filter_range(rank: int, filters_per_rank: int) -> tuple[int, int]:
    """Global indices [first, last) of rank's filters."""
    return rank * filters_per_rank, (rank + 1) * filters_per_rank


def rng_counter(rank: int) -> tuple[int, int]:
    """Start counter of rank's fills: blocks (i, rank), i < 2^32, disjoint
    from every other rank's as long as one rank draws fewer than 2^32
    blocks (the engine carries into the second word only past that)."""
    return (0, rank)


def job_rate(units: float, seconds: float, world: int, device=None) -> tuple[float, float]:
    """(units summed over ranks / max seconds over ranks, max seconds).
    Every rank must call it at the same point (two all-reduces)."""
    if world == 1:
        return units / seconds, seconds
    import torch
    import torch.distributed as dist

    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(u.item()) / float(t.item()), float(t.item())
