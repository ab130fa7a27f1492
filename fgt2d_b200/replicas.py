"""Multi-GPU plumbing for independent replicas (one process per GPU).

The transform does not shard across GPUs here: each rank runs its own
problem, and the whole-job rate is the sum of the ranks' points over the
slowest rank's time.  These helpers are what bench.py uses; they work on any
torch.distributed backend (NCCL on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations


def _device_for(backend: str):
    import torch
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """Maximum of ``x`` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for(dist.get_backend()))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for(dist.get_backend()))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def whole_job_rate(points_this_rank: float, seconds_this_rank: float) -> float:
    """Sum of points over ranks / max of seconds over ranks."""
    return sum_over_ranks(points_this_rank) / max_over_ranks(seconds_this_rank)


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's replica: distinct per rank, fixed per run."""
    return base + 7919 * rank
