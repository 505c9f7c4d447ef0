"""Sharding of runs over ranks (one process per GPU).

Runs are independent and keyed by (seed, run index), so a job splits into
disjoint run ranges with no data-path exchange: rank r of W simulates, for
step s, the runs [(s*W + r)*n, (s*W + r + 1)*n).  Only the per-rank totals
are combined: counters by a sum, times by a maximum (the slowest rank sets
the job's time).  With torch.distributed over NCCL this is one small
all-reduce per quantity at the end of a timed region.
"""
from __future__ import annotations


def first_run(step: int, rank: int, world: int, runs_per_rank: int) -> int:
    """First run index of rank's range in a step."""
    return (step * world + rank) * runs_per_rank


def combine(counters, times, device=None):
    """Sums the integer counters and takes the maximum of the times over all
    ranks of the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(counters), list(times)
    c = torch.tensor(list(counters), dtype=torch.int64, device=device)
    t = torch.tensor(list(times), dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return c.tolist(), t.tolist()
