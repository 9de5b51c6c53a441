"""Several processes (one per GPU) over torch.distributed.

The scan needs no exchange between GPUs: each rank either runs its own replica of the
whole workload (how bench.py runs N GPUs: weak scaling) or owns a contiguous partition of
the windows, as the reference's ranks own chunks of the record (Tremor.cpp:3773-3794,
replication.cpp:264-275). A partition is set on a context with
Context.set_window_range(first, count); the rank's threshold hits are its shard (the
reference writes one CSV shard per rank and merges within a shard, SkipSequential.cpp:
358-370; validate_search.py:136-148 checks exactly that), so no collective is needed for
threshold answers. kNN over partitions needs one exchange, as in the reference
(Tremor.cpp:337-408): each rank's candidates (knn_candidates) are gathered and every rank
makes the canonical selection over their union (select_knn, knn_partitioned). The other
collective is the report: total work and the slowest rank's time.
"""
from __future__ import annotations

import bisect
from typing import List, Sequence, Tuple

import numpy as np

FLT_MAX = float(np.finfo(np.float32).max)


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


def knn_candidates(ctx, templates: Sequence[np.ndarray], k: int, merge_offset: int) -> List[Tuple[np.ndarray, np.ndarray]]:
    """This rank's share of the kNN candidates of each template, (positions, distances),
    for the canonical answer over all ranks' partitions (Tremor.cpp:139-149).

    Without an exclusion zone the rank's k nearest windows are its candidates. With one,
    the rank's canonical answer for 2k - 1 (a set of windows pairwise at least
    merge_offset apart) bounds the k-th distance of the answer over all ranks: each of the
    first k - 1 answers excludes at most 2 of those windows, so one is left for the k-th.
    Every window of the partition within that bound is a candidate; a rank with fewer
    than 2k - 1 separated windows gives every window of its partition. The bound's windows
    come from a threshold search (merge 0) with a correlation a few float ulps below the
    bound's, so the search is a superset; the candidates are then the hits at or below
    the bound, compared on the returned FP32 distance bits."""
    from tremor_b200 import MODE_KNN, MODE_THRESHOLD, Request
    ts = [np.ascontiguousarray(t, dtype=np.float32) for t in templates]
    if not ts:
        return []
    wide = 2 * k - 1 if merge_offset > 0 else k
    local = ctx.scan_batch([Request(t, MODE_KNN, k=wide, merge_offset=merge_offset) for t in ts])
    if merge_offset <= 0:
        return [(p[d < FLT_MAX].copy(), d[d < FLT_MAX].copy()) for p, d in local]
    bounds, reqs = [], []
    for t, (_, d) in zip(ts, local):
        m = len(t)
        tau = float(d.max()) if len(d) and d.max() < FLT_MAX else float('inf')
        bounds.append(tau)
        if np.isfinite(tau):
            ed = tau * (1.0 + 1e-4) + 2.0 * m * 2.0 ** -20
            corr = max(1.0 - ed / (2.0 * m), -2.0)
        else:
            corr = -2.0  # every window with a finite distance (z-normalised distances are <= 4m)
        reqs.append(Request(t, MODE_THRESHOLD, correlation=corr, merge_offset=0))
    out = []
    for tau, (p, d) in zip(bounds, ctx.scan_batch(reqs)):
        keep = (d <= np.float32(tau)) & (d < FLT_MAX) if np.isfinite(tau) else d < FLT_MAX
        out.append((p[keep].copy(), d[keep].copy()))
    return out


def select_knn(positions: np.ndarray, distances: np.ndarray, k: int, merge_offset: int) -> Tuple[np.ndarray, np.ndarray]:
    """The canonical exclusion-zone selection (ZnormSearch.hpp:170-189): candidates by
    (distance, position); a window is kept unless it lies less than merge_offset from one
    already kept, until k are kept. Returns k (positions, distances), missing answers as
    (0, FLT_MAX) (Tremor.cpp:400-404)."""
    pos = np.asarray(positions, np.uint64)
    dist = np.asarray(distances, np.float32)
    order = np.lexsort((pos, dist))
    kept_sorted: List[int] = []
    out_p = np.zeros(k, np.uint64)
    out_d = np.full(k, FLT_MAX, np.float32)
    n = 0
    for i in order:
        if n == k:
            break
        p = int(pos[i])
        j = bisect.bisect_left(kept_sorted, p)
        if j < len(kept_sorted) and kept_sorted[j] - p < merge_offset:
            continue
        if j > 0 and p - kept_sorted[j - 1] < merge_offset:
            continue
        kept_sorted.insert(j, p)
        out_p[n], out_d[n] = p, dist[i]
        n += 1
    return out_p, out_d


def knn_partitioned(ctx, templates: Sequence[np.ndarray], k: int, merge_offset: int = 0,
                    dist=None) -> Tuple[np.ndarray, np.ndarray]:
    """kNN over the windows of all ranks, each rank searching its own partition (its
    context's window range): the candidates of every rank gathered on every rank and the
    canonical selection made there (Tremor.cpp:337-408, which gathers on rank 0 and
    broadcasts the answer; every rank computes the same answer here). Returns (I, D) of
    shape (templates, k), as Context.search_knn. Every rank calls it with the same
    templates (the same collective in the same order)."""
    mine = knn_candidates(ctx, templates, k, merge_offset)
    shards = gather_shards([(p.tolist(), d.tolist()) for p, d in mine], dist)
    I = np.zeros((len(mine), k), np.uint64)
    D = np.full((len(mine), k), FLT_MAX, np.float32)
    for q in range(len(mine)):
        p = np.concatenate([np.asarray(s[q][0], np.uint64) for s in shards])
        d = np.concatenate([np.asarray(s[q][1], np.float32) for s in shards])
        I[q], D[q] = select_knn(p, d, k, merge_offset)
    return I, D
