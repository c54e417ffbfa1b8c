"""Multi-GPU replicas (one process per GPU, weak scaling).

Products are independent, so N GPUs run N independent batches: rank r works
on the seeded batch of replicate 1 + r, no data crosses between ranks, and
the only collectives are the timing barrier and the maximum of the per-rank
times.  Throughput = units of all ranks / slowest rank's time.
"""
from __future__ import annotations

from datetime import timedelta


def replicate_of(rank: int) -> int:
    """Seed replicate of a rank's batch (rank 0 reproduces the golden batch)."""
    return 1 + rank


def init(backend: str, rank: int, world: int, device=None, timeout_s: int = 120):
    """Process group for timing only (barrier + max); returns the module."""
    import torch.distributed as dist
    kw = {"timeout": timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, rank=rank, world_size=world, **kw)
    return dist


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank value (e.g. elapsed milliseconds)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, steps: int, max_ms: float) -> float:
    """Units per second of the whole job, timed by its slowest rank."""
    return units_per_rank * world * steps / (max_ms / 1000.0)
