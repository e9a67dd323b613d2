"""
Multi-GPU runs of independent volumes: one process per GPU, each evaluating its own volumes
(replicas), so the path needs no data-path collective.  The only exchange is the
max-over-ranks of the timed region, from which the whole-job throughput follows.
"""

from __future__ import annotations

import os


def rank_env():
    """(rank, world_size, local_rank) from the torchrun environment (0, 1, 0 without one)."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def slowest(seconds, device=None):
    """The largest of every rank's time (seconds); the local value without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(units_per_rank, seconds, world):
    """Whole-job rate: every rank's units over the slowest rank's time."""
    return world * units_per_rank / seconds if seconds > 0 else float("nan")
