"""Multi-GPU plumbing for independent chain replicas (one process per GPU).

The sampler's chains are independent (RWM, MALA; a PT ladder and a DE pool
live inside one replica), so N GPUs run N replicas with no data-path
collective: each rank gets its own chain streams (its seed offset by the
rank), times its own iterations on the device, and only the device times
meet in one MAX reduction so the whole-job rate is units over the slowest
rank.  The functions take a ``torch.distributed`` process group that is
already initialised (NCCL on GPUs; gloo works the same for the host logic).
"""
from __future__ import annotations

import os


def rank_env():
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base: int, rank: int) -> int:
    """Seed of a replica: distinct per rank, so replicas draw independent streams."""
    return (int(base) + int(rank)) & 0xFFFFFFFF


def max_over_ranks(seconds: float, device=None) -> float:
    """The largest of the ranks' values (device times), on every rank."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Units processed by all ranks per second of the slowest rank (weak scaling)."""
    if not max_seconds > 0:
        raise ValueError("max_seconds must be positive")
    return world * float(units_per_rank) / float(max_seconds)
