"""Replicas across GPUs: the increment does not shard (one bar per GPU), so N processes run N
independent bars and the job's throughput is the sum over them, timed by the slowest rank.
The reduction works on any torch.distributed backend (NCCL on the GPUs, gloo on CPU)."""
from __future__ import annotations


def max_over_ranks(x: float, device=None) -> float:
    """Largest x over the ranks of the default process group (x itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    if device is None:
        device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(points_per_rank: int, steps: int, slowest_ms: float, world: int) -> float:
    """Particle-steps/s of the whole job: every rank advances its own bar by `steps`
    increments, and the job is done when the slowest rank is."""
    return world * points_per_rank * steps / (slowest_ms * 1e-3)
