"""Multi-GPU runs of the path: independent replicas, one process per GPU.

Paths are independent, so every rank renders its own copy of the workload with no data-path
collective; the only communication is the timing reduction. The job's time is the slowest
rank's (max over ranks), and its throughput counts the paths of all ranks.
"""

from __future__ import annotations


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks of the default process group (itself when there is
    none). `device` places the reduction tensor (a CUDA device under NCCL, None = CPU for gloo)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(paths_per_rank_step: int, steps: int, world: int, job_seconds: float) -> float:
    """Whole-job Mpaths/s: the paths of all `world` ranks over the slowest rank's time."""
    if job_seconds <= 0:
        raise ValueError("job time must be positive")
    return world * paths_per_rank_step * steps / job_seconds / 1e6
