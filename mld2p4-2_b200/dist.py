"""Multi-GPU plumbing for independent solves (one process per GPU).

The benchmarked forms have no exchange step: every system (or every
right-hand-side column block) is an independent unit.  Units are dealt to
ranks round-robin by index, each rank solves its own units on its own GPU, and
only statistics cross ranks: the timed region is closed by a barrier and the
device times are reduced with MAX (the job's time is its slowest rank).
Works with any torch.distributed backend (nccl on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

from typing import Sequence


def shard(units: Sequence, rank: int, world: int) -> list:
    """Units owned by `rank`: indices rank, rank+world, ... (deterministic)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"bad rank/world {rank}/{world}")
    return [u for i, u in enumerate(units) if i % world == rank]


def owner(index: int, world: int) -> int:
    return index % world


def max_over_ranks(value: float, device=None) -> float:
    """MAX-reduce a per-rank device time (no-op without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_throughput(units_per_rank: int, world: int, max_ms: float) -> float:
    """Whole-job units per second: all ranks' units over the slowest rank's time."""
    return units_per_rank * world / (max_ms * 1e-3)
