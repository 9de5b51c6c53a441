"""Several processes (one per GPU) over torch.distributed.

The scan needs no exchange between GPUs: each rank either runs its own replica of the
whole workload (how bench.py runs N GPUs: weak scaling) or owns a contiguous partition of
the windows, as the reference's ranks own chunks of the record (Tremor.cpp:3773-3794,
replication.cpp:264-275). A partition is set on a context with
Context.set_window_range(first, count); the rank's threshold hits are its shard (the
reference writes one CSV shard per rank and merges within a shard, SkipSequential.cpp:
358-370; validate_search.py:136-148 checks exactly that), so no collective is needed for
answers either. The only collective is the report: total work and the slowest rank's
time.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def partition(windows: int, world: int, rank: int) -> Tuple[int, int]:
    """(first, count) of rank's contiguous share of `windows` windows (sizes differ by at
    most one; the shares tile [0, windows))."""
    if world < 1 or not 0 <= rank < world or windows < 0:
        raise ValueError('invalid partition request')
    base, extra = divmod(windows, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def combine(work: float, milliseconds: float, dist=None, device=None) -> Tuple[float, float]:
    """(total work over all ranks, the slowest rank's milliseconds): every rank calls it
    (the same collectives in the same order); without a process group, the local values."""
    if dist is None:
        return work, milliseconds
    import torch
    t = torch.tensor([work, milliseconds], dtype=torch.float64, device=device)
    total = t.clone()
    dist.all_reduce(total, op=dist.ReduceOp.SUM)
    slowest = t.clone()
    dist.all_reduce(slowest, op=dist.ReduceOp.MAX)
    return float(total[0]), float(slowest[1])


def gather_shards(shard: Sequence, dist=None) -> List:
    """Every rank's shard (any picklable value), in rank order, on every rank."""
    if dist is None:
        return [shard]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, shard)
    return out
