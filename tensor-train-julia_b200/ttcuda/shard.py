"""Batch sharding across GPUs (one process per GPU, weak scaling).

A single TT rounding is sequential over its sites and does not shard; a batch of independent
TTs does.  Each rank owns its own batch (inputs generated or uploaded per rank), rounds it with
no data-path collective, and the job's time is the maximum over ranks of the device-measured
time.  These helpers hold that host logic so that it is the same in the benchmark and in the
multi-process tests.
"""
from __future__ import annotations

from typing import Optional, Sequence


def rank_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s synthetic batch: distinct and reproducible per rank."""
    return int(base) + int(rank)


def shard_indices(count: int, rank: int, world: int) -> Sequence[int]:
    """Indices of a shared list of `count` TTs that rank `rank` of `world` rounds: contiguous,
    sizes differing by at most one."""
    base, extra = divmod(int(count), int(world))
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, dist=None, device: Optional[str] = None) -> float:
    """Maximum of `value` over the process group (the value itself without one).  `device` is
    where the reduction tensor lives: a CUDA device for NCCL, "cpu" for gloo."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, steps: int, ms: float) -> float:
    """Units per second of the whole job: all ranks' units over the max-over-ranks time."""
    return float(units_per_rank) * int(world) * int(steps) / (float(ms) / 1e3)
