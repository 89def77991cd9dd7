"""Several GPUs: one process per GPU, each running its own replica of the substep.

The substep of one coupled scene does not shard (contacts and the global solve couple every
vertex with its neighbours at every ADMM iteration), so N GPUs run N independent replicas: the
same scene, or for a batch of bodies each rank its own batch (``rank_seed``).  There is no
collective on the data path; the only communication is the timing reduction below, which takes
the slowest rank's device time as the job's time, over NCCL on GPUs or gloo on the CPU.
"""
from __future__ import annotations

from typing import Optional


def rank_seed(base_seed: int, rank: int) -> int:
    """Seed of a rank's own batch of bodies."""
    return int(base_seed) + int(rank)


def max_over_ranks(value: float, device: Optional[str] = None) -> float:
    """The maximum of `value` over the ranks of the default process group (the value itself
    without one).  `device`: where the reduction tensor lives (``cuda:k`` for NCCL, CPU for
    gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(steps_per_rank: int, world: int, max_seconds: float) -> float:
    """Whole-job substeps per second: every rank ran `steps_per_rank` substeps, the job took the
    slowest rank's time."""
    return world * steps_per_rank / max_seconds
