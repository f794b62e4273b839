"""Independent replicas across ranks (one process per GPU).

The directional FMM matvec does not shard: a distributed FMM would need
per-level exchanges that the method (and the reference) does not have.  On N
GPUs each rank therefore runs its own problem -- the same workload with its
own seeded charges -- and the ranks meet only to time the job: a barrier on
both sides of the timed region and the maximum of the per-rank times.  No
collective touches the data path.
"""
from __future__ import annotations


def replica_seed(rank: int, base: int = 1) -> int:
    """Seed of the charge vector of a rank's replica."""
    return base + rank


def job_throughput(points_per_replica: int, world: int, max_seconds: float) -> float:
    """Whole-job points/s: all replicas' points over the slowest rank's time."""
    return world * points_per_replica / max_seconds


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """Maximum of a per-rank scalar (identity without a process group)."""
    if dist is None or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
