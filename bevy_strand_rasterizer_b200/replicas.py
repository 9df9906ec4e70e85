"""Replica scaling: one process per GPU, each rendering its own frames.

Frames, views and requests are independent, so N GPUs run N replicas with no
collective on the data path. The only collective is the timing reduction: the
job's time is the slowest rank's device time, and its throughput is the units
all ranks processed divided by that time.
"""
from __future__ import annotations

FRAME_STRIDE = 100_003  # orbit frames of rank r start at r * FRAME_STRIDE


def frame_index(rank: int, k: int) -> int:
    """Frame k of replica `rank` (disjoint across ranks for k < FRAME_STRIDE)."""
    return rank * FRAME_STRIDE + k


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over the default process group (itself when no
    group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return units_per_rank * world / max_seconds
