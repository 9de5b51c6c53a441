"""Several ranks (tremor_b200.replicas) on CPU with the gloo backend, world size 2: the
report's combination (total work, slowest rank), the contiguous window partitions, and the
threshold shards of a partitioned search (each rank's oracle answers over its partition,
gathered in rank order) against the whole record's answers."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tremor_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, x, q, m, corr, merge, out):
    import datetime
    import torch.distributed as dist
    from tests import oracle_bindings as ob
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        total, slowest = replicas.combine(1000.0 + rank, 10.0 * (rank + 1), dist)
        W = len(x) - m + 1
        first, count = replicas.partition(W, world, rank)
        part = x[first:first + count + m - 1]                 # the partition and its m - 1 halo
        _, pos, dist_ed = ob.scan_threshold(part, q[None, :], m, corr, merge)
        shard = [(int(p) + first, float(d)) for p, d in zip(pos, dist_ed)]
        shards = replicas.gather_shards(shard, dist)
        out.put((rank, total, slowest, (first, count), shards))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('merge', [0, 25])
def test_two_ranks_partitioned_threshold_search(merge):
    rng = np.random.default_rng(5 + merge)
    n, m, corr = 6000, 64, 0.5
    x = rng.normal(size=n).astype(np.float32)
    q = x[1000:1000 + m].copy()
    x[2990:2990 + m] = q          # a match across the partition boundary region
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, x, q, m, corr, merge, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, total0, slow0, part0, shards0), (r1, total1, slow1, part1, shards1) = results
    assert total0 == total1 == 2001.0 and slow0 == slow1 == 20.0
    W = n - m + 1
    assert part0 == (0, (W + 1) // 2) and part1 == ((W + 1) // 2, W // 2)
    assert shards0 == shards1 and len(shards0) == 2
    from tests import oracle_bindings as ob
    gathered = [h for shard in shards0 for h in shard]
    expected = []
    for first, count in (part0, part1):          # the reference merges within each rank's shard
        _, pos, d = ob.scan_threshold(x[first:first + count + m - 1], q[None, :], m, corr, merge)
        expected += [(int(p) + first, float(v)) for p, v in zip(pos, d)]
    assert gathered == expected
    if merge == 0:                                # no merge: exactly the whole record's hits
        _, pos, d = ob.scan_threshold(x, q[None, :], m, corr, 0)
        assert gathered == [(int(p), float(v)) for p, v in zip(pos, d)]
    assert any(p == 2990 for p, _ in gathered)


def test_partition_tiles_the_windows():
    for windows in (0, 1, 7, 1000, 12345):
        for world in (1, 2, 3, 8):
            parts = [replicas.partition(windows, world, r) for r in range(world)]
            assert parts[0][0] == 0 and sum(c for _, c in parts) == windows
            for (f0, c0), (f1, _) in zip(parts, parts[1:]):
                assert f0 + c0 == f1
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1
    with pytest.raises(ValueError):
        replicas.partition(10, 2, 2)


class _OracleContext:
    """A context over one rank's partition (the windows [first, first + count) and their
    m - 1 halo) whose scan_batch answers through the oracle: the host logic of the
    partitioned kNN under test, with the oracle standing in for the device search."""

    def __init__(self, x, first, count, m):
        self.part, self.first, self.m = x[first:first + count + m - 1], first, m

    def scan_batch(self, requests):
        import tremor_b200 as tb
        from tests import oracle_bindings as ob
        out = []
        for r in requests:
            if r.mode == tb.MODE_KNN:
                I, D = ob.scan_knn(self.part, r.template[None, :], self.m, r.k, r.merge_offset)
                pos = np.where(D[0] < ob.FLT_MAX, I[0] + np.uint64(self.first), 0).astype(np.uint64)
                out.append((pos, D[0]))
            else:
                _, pos, d = ob.scan_threshold(self.part, r.template[None, :], self.m, r.correlation, r.merge_offset)
                out.append((pos.astype(np.uint64) + np.uint64(self.first), d))
        return out


def _knn_rank_main(rank, world, port, x, q, m, k, merge, out):
    import datetime
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first, count = replicas.partition(len(x) - m + 1, world, rank)
        I, D = replicas.knn_partitioned(_OracleContext(x, first, count, m), list(q), k, merge, dist)
        out.put((rank, I, D))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('n,m,k,merge', [(6000, 64, 5, 0), (6000, 64, 5, 40), (6000, 64, 3, 200), (600, 32, 10, 50), (600, 32, 14, 50)])
def test_two_ranks_partitioned_knn_equals_whole_record(n, m, k, merge):
    """knn_partitioned over two gloo ranks equals the oracle's kNN over the whole record,
    with near-copies of a template planted on both sides of the partition boundary (each
    rank keeps its own; over the whole record the nearer one excludes the other) and, in
    the last cases, partitions too short for 2k - 1 separated windows (every window is a
    candidate; answers padded where k do not fit)."""
    from tests import oracle_bindings as ob
    rng = np.random.default_rng(n + k + merge)
    x = rng.normal(size=n).astype(np.float32)
    q = np.stack([x[100:100 + m].copy(), rng.normal(size=m).astype(np.float32)])
    boundary = replicas.partition(n - m + 1, 2, 1)[0]
    left, right = boundary - m - 3, boundary + 2       # m + 5 apart, one in each partition
    x[left:left + m] = q[0] + 0.01 * rng.normal(size=m).astype(np.float32)
    x[right:right + m] = q[0] + 0.001 * rng.normal(size=m).astype(np.float32)
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_knn_rank_main, args=(r, 2, port, x, q, m, k, merge, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted((out.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    Io, Do = ob.scan_knn(x, q, m, k, merge)
    Io = np.where(Do < ob.FLT_MAX, Io, 0)
    for _, I, D in results:
        assert np.array_equal(I, Io) and np.array_equal(D.view(np.uint32), Do.view(np.uint32)), (I, Io, D, Do)
    if n == 6000:
        assert right in Io[0] and (left in Io[0]) == (merge <= m + 5)
    if n == 600:  # no rank has 2k - 1 windows merge apart: every window is a candidate
        assert (n - m + 1) // 2 < (2 * k - 2) * merge
    if k == 14:   # more answers asked for than fit merge apart: padding
        assert np.any(Do >= ob.FLT_MAX)


def test_select_knn_is_the_canonical_selection():
    """select_knn against the oracle's kNN on random distance profiles: the candidates
    are every window, so the selection must equal the whole scan's answer."""
    from tests import oracle_bindings as ob
    rng = np.random.default_rng(3)
    x = rng.normal(size=3000).astype(np.float32)
    m = 48
    q = rng.normal(size=m).astype(np.float32)
    prof = ob.distance_profile(x, q, m)
    for k, merge in ((1, 0), (7, 0), (7, 24), (20, 100)):
        I, D = replicas.select_knn(np.arange(len(prof), dtype=np.uint64), prof, k, merge)
        Io, Do = ob.scan_knn(x, q[None, :], m, k, merge)
        assert np.array_equal(I, np.where(Do[0] < ob.FLT_MAX, Io[0], 0))
        assert np.array_equal(D.view(np.uint32), Do[0].view(np.uint32))
