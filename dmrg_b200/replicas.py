"""Replica timing across ranks (one process per GPU, no data-path collective).

The matvec does not shard profitably, so N GPUs run N independent replicas.  A
job's throughput is the total work over the slowest rank's device time; the
only collective is this one scalar reduction, on whatever backend the process
group uses (NCCL on GPUs, gloo in the CPU tests)."""
from __future__ import annotations


def max_over_ranks(x: float, device=None) -> float:
    """The maximum of a per-rank float over all ranks (x itself without a group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: int, seconds: float, device=None) -> float:
    """Whole-job rate: units over all ranks / the slowest rank's seconds."""
    import torch.distributed as dist
    world = dist.get_world_size() if (dist.is_available() and dist.is_initialized()) else 1
    return world * units_per_rank / max_over_ranks(seconds, device)
