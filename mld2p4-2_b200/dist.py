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


def deal_balanced(weights: Sequence[float], world: int) -> list:
    """Indices of the units each rank owns, balancing the summed weight:
    units taken in decreasing weight (ties by index) go to the rank with the
    smallest load so far (ties by rank).  Deterministic: every rank computes
    the same dealing.  Returns world lists of ascending indices."""
    if world < 1:
        raise ValueError(f"bad world {world}")
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda k: (-float(weights[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += float(weights[i])
    return [sorted(p) for p in parts]


def column_block(ncols: int, rank: int, world: int) -> tuple:
    """Contiguous column range [lo, hi) of `rank` (blocks differ by at most one)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"bad rank/world {rank}/{world}")
    return ncols * rank // world, ncols * (rank + 1) // world


def merge_results(owned: Sequence[int], results: Sequence, total: int) -> list:
    """Gather every rank's (unit index -> result) into one list in unit order,
    on every rank (all_gather_object; the local list without a process
    group).  Raises if a unit is missing or owned twice."""
    import torch.distributed as dist
    if len(owned) != len(results):
        raise ValueError("one result per owned unit")
    pairs = list(zip([int(i) for i in owned], results))
    if dist.is_available() and dist.is_initialized():
        allp = [None] * dist.get_world_size()
        dist.all_gather_object(allp, pairs)
        pairs = [p for part in allp for p in part]
    out = [None] * total
    for i, v in pairs:
        if not (0 <= i < total) or out[i] is not None:
            raise ValueError(f"unit {i} out of range or owned twice")
        out[i] = v
    if any(v is None for v in out):
        raise ValueError("a unit has no result")
    return out
