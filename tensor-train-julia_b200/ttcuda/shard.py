"""Batch sharding across GPUs (one process per GPU, no data-path collective).

A single TT rounding is sequential over its sites and does not shard; a batch of independent
TTs does.  All ranks know the whole batch's shape (its rank lists), partition it by estimated
work, and each rank uploads and rounds only its own TTs; the job's time is the maximum over
ranks of the device-measured time, so the partition must balance work, not counts: the TTs of
a batch have uneven ranks (config 3 draws them from U[16,256]) and a rounding's cost grows like
the cube of its bond ranks.  These helpers hold that host logic so that it is the same in the
benchmark and in the multi-process tests.
"""
from __future__ import annotations

import heapq
from typing import List, Optional, Sequence


def rank_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s synthetic batch when ranks generate independent batches."""
    return int(base) + int(rank)


def tt_work(ranks: Sequence[int]) -> float:
    """Estimated work of rounding one TT: sum over bonds of r_k^3 (QR, SVD and contractions of a
    site all scale with the cube of its bond ranks)."""
    return float(sum(int(r) ** 3 for r in ranks))


def shard_by_work(works: Sequence[float], world: int) -> List[List[int]]:
    """Greedy partition of a batch over `world` ranks: TTs in decreasing order of work, each to
    the rank with the least work so far (ties to the lower rank).  Returns each rank's indices in
    increasing order.  The largest shard is within max(works) of the ideal share."""
    world = int(world)
    heap = [(0.0, r) for r in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(works)), key=lambda j: (-float(works[j]), j)):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(works[i]), r))
    return [sorted(s) for s in shards]


def shard_indices(count: int, rank: int, world: int) -> Sequence[int]:
    """Contiguous split of `count` items by count (sizes differ by at most one), for batches whose
    items cost the same."""
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


def job_rate(units_total: int, steps: int, ms: float) -> float:
    """Units per second of a job of `units_total` units per step over the max-over-ranks time."""
    return float(units_total) * int(steps) / (float(ms) / 1e3)
