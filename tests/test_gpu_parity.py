"""GPU parity: the CUDA path against the reference's answers and the pinned oracle.

Every case compares through the C ABI (tremor_b200.Context -> libtremor_b200.so):
  * golden fixtures (answers printed by the reference's own SkipSequentialScan):
    identical CSV rows, for every contraction kernel;
  * random cases against the oracle (bit-identical to the reference's kernels):
    identical answer positions and bit-identical FP32 distances, with missing
    samples, constant stretches, loud/quiet stretches, m % 32 tails, exclusion zones
    wider than a kNN bucket, and thresholds with many hits;
  * the reference's per-window statistics, bit for bit.
Tolerance: none. Integer positions and FP32 distances must match exactly; the FP64
check of test_oracle.py (correlation within 2e-4 of FP64) then carries over.
"""
import numpy as np
import pytest

import tremor_b200 as tb
from tests import oracle_bindings as ob

pytestmark = pytest.mark.gpu

KERNELS = [tb.KERNEL_FP32, tb.KERNEL_AUTO]


def _ctx(x, kernel):
    ctx = tb.Context(x)
    ctx.set_kernel(kernel)
    return ctx


@pytest.mark.parametrize('kernel', KERNELS)
@pytest.mark.parametrize('name', ob.golden_cases())
def test_golden_cases(name, kernel):
    meta, x, q = ob.load_golden(name)
    m = meta['m']
    with _ctx(x, kernel) as ctx:
        for merge in meta['merges']:
            I, D = ctx.search_knn(q, meta['k'], merge)
            assert tb.knn_rows(I, D, m) == meta['knn'][str(merge)], (name, merge)
            hits = ctx.search_threshold(q, meta['threshold'], merge)
            assert tb.threshold_rows(hits, m) == meta['threshold_hits'][str(merge)], (name, merge)


def _waveform(n, seed):
    from tremor_b200 import synth
    rng = np.random.default_rng(seed)
    x = synth.ar2_waveform(n, rng) + np.float32(3.0)  # with an offset
    x[1000:1000 + 3000] = 2.0                      # constant stretch
    x[20000:24000] *= np.float32(1e5)              # loud
    x[24000:30000] *= np.float32(1e-4)             # quiet after loud
    x[rng.integers(0, n, 50)] = tb.MISSING_VALUE   # scattered missing samples
    x[50000:50100] = tb.MISSING_VALUE              # a gap
    return x


def _templates(x, m, rng, count):
    from tremor_b200 import synth
    out = [x[p:p + m].copy() for p in rng.integers(0, len(x) - m, count // 2)]
    out += list(synth.chirp_templates(count - len(out), m, rng))
    q = np.stack(out).astype(np.float32)
    q[q == tb.MISSING_VALUE] = 0.0
    return q


def _assert_knn_equal(x, q, m, k, merge, I, D):
    Io, Do = ob.scan_knn(x, q, m, k, merge)
    assert np.array_equal(I, Io), (m, k, merge)
    assert np.array_equal(D.view(np.uint32), Do.view(np.uint32)), (m, k, merge)


@pytest.mark.parametrize('kernel', KERNELS)
@pytest.mark.parametrize('m', [48, 100, 256, 1000])
def test_random_knn_matches_oracle(kernel, m):
    x = _waveform(1 << 17, 7 + m)
    rng = np.random.default_rng(m)
    q = _templates(x, m, rng, 6)
    with _ctx(x, kernel) as ctx:
        for k, merge in [(1, 0), (5, m // 2), (40, 0), (7, 3000)]:
            I, D = ctx.search_knn(q, k, merge)
            _assert_knn_equal(x, q, m, k, merge, I, D)


@pytest.mark.parametrize('m', [150, 300, 384, 520])
def test_fp32_stage_depths(m):
    """The FP32 kernel's two stage depths: padded lengths 192 and 320 (stages of 64
    samples, several of them) and 384 and 576 (stages of 128 when the padded length is a
    multiple of 128, else 64), against the oracle bit for bit."""
    x = _waveform(1 << 16, 31 + m)
    q = _templates(x, m, np.random.default_rng(m + 3), 4)
    with _ctx(x, tb.KERNEL_FP32) as ctx:
        for k, merge in [(1, 0), (6, m // 2)]:
            I, D = ctx.search_knn(q, k, merge)
            _assert_knn_equal(x, q, m, k, merge, I, D)


@pytest.mark.parametrize('kernel', KERNELS)
@pytest.mark.parametrize('m', [48, 256, 1000])
def test_random_threshold_matches_oracle(kernel, m):
    x = _waveform(1 << 17, 100 + m)
    rng = np.random.default_rng(m + 1)
    q = _templates(x, m, rng, 6)
    with _ctx(x, kernel) as ctx:
        for corr, merge in [(0.3, 0), (0.6, 25), (0.9, 0)]:
            hits = ctx.search_threshold(q, corr, merge)
            qid, pos, dist = ob.scan_threshold(x, q, m, corr, merge)
            for i, (p, d) in enumerate(hits):
                assert np.array_equal(p, pos[qid == i]), (m, corr, merge, i)
                assert np.array_equal(d.view(np.uint32), dist[qid == i].view(np.uint32))


def test_window_stats_bit_identical():
    x = _waveform(1 << 16, 3)
    with tb.Context(x) as ctx:
        for m in [32, 72, 1000]:
            mean, std = ctx.window_stats(m)
            W = len(x) - m + 1
            mo, so = np.zeros(W, np.float32), np.zeros(W, np.float32)
            ob.oracle().tmo_window_stats(ob.P(x), W, m, ob.P(mo), ob.P(so))
            assert np.array_equal(mean.view(np.uint32), mo.view(np.uint32))
            assert np.array_equal(std.view(np.uint32), so.view(np.uint32))


@pytest.mark.parametrize('kernel', KERNELS)
def test_mixed_batch_equals_single_requests(kernel):
    x = _waveform(1 << 16, 11)
    rng = np.random.default_rng(12)
    reqs = []
    for m in [64, 200, 64, 512]:
        q = _templates(x, m, rng, 2)
        reqs.append(tb.Request(q[0], tb.MODE_KNN, k=5, merge_offset=m // 2))
        reqs.append(tb.Request(q[1], tb.MODE_THRESHOLD, correlation=0.5, merge_offset=10))
    with _ctx(x, kernel) as ctx:
        together = ctx.scan_batch(reqs)
        for r, (p, d) in zip(reqs, together):
            alone = ctx.scan_batch([r])[0]
            assert np.array_equal(p, alone[0]) and np.array_equal(d.view(np.uint32), alone[1].view(np.uint32))


@pytest.mark.parametrize('kernel', KERNELS)
def test_window_range_is_a_partition(kernel):
    """tm_set_window_range = one data partition (SkipSequential.cpp:218-226)."""
    x = _waveform(1 << 16, 21)
    m, first, count = 128, 12345, 30000
    q = _templates(x, m, np.random.default_rng(22), 3)
    part = x[first:first + count + m - 1].copy()
    with _ctx(x, kernel) as ctx:
        ctx.set_window_range(first, count)
        I, D = ctx.search_knn(q, 6, 64)
        Io, Do = ob.scan_knn(part, q, m, 6, 64)
        assert np.array_equal(I, np.where(Do < ob.FLT_MAX, Io + first, 0))
        assert np.array_equal(D.view(np.uint32), Do.view(np.uint32))


@pytest.mark.parametrize('merge', [0, 64, 700])
def test_partitioned_knn_equals_whole_record(merge):
    """kNN over three window partitions (one context each, as three ranks would hold
    them): every partition's candidates (replicas.knn_candidates, two device searches)
    and the canonical selection over their union equal the whole record's kNN, with
    near-copies of a template planted on both sides of each partition boundary."""
    from tremor_b200 import replicas
    x = _waveform(1 << 16, 23)
    m, k = 128, 10
    rng = np.random.default_rng(24)
    q = _templates(x, m, rng, 3)
    W = len(x) - m + 1
    parts = [replicas.partition(W, 3, r) for r in range(3)]
    for first, _ in parts[1:]:  # m + 5 apart, one on each side of the boundary
        for off, eps in ((-m - 3, 0.02), (2, 0.005)):
            x[first + off:first + off + m] = q[0] + eps * np.std(q[0]) * rng.normal(size=m).astype(np.float32)
    with tb.Context(x) as whole:
        I, D = whole.search_knn(q, k, merge)
    cands = []
    for first, count in parts:
        with tb.Context(x) as ctx:
            ctx.set_window_range(first, count)
            cands.append(replicas.knn_candidates(ctx, list(q), k, merge))
    for i in range(len(q)):
        p = np.concatenate([c[i][0] for c in cands])
        d = np.concatenate([c[i][1] for c in cands])
        Ip, Dp = replicas.select_knn(p, d, k, merge)
        assert np.array_equal(Ip, I[i]) and np.array_equal(Dp.view(np.uint32), D[i].view(np.uint32)), (merge, i)
    for first, _ in parts[1:]:
        assert first + 2 in I[0] and (first - m - 3 in I[0]) == (merge <= m + 5)


@pytest.mark.parametrize('kernel', KERNELS)
def test_config1_shape_self_match_and_oracle(kernel):
    """The plain kNN workload's shape (2^22 samples, m=1024, k=10, merge m/2): planted
    exact copies are found first with distance ~0, and two templates match the oracle."""
    from tremor_b200 import synth
    x, q, _ = synth.workload(1 << 22, 16, 1024, 50, seed=2026)
    rng = np.random.default_rng(1)
    planted = rng.integers(0, len(x) - 1024, 16)
    for i, p in enumerate(planted):  # scaled, offset exact copies: correlation 1
        x[p:p + 1024] = q[i] * np.float32(3.0) + np.float32(0.5)
    with _ctx(x, kernel) as ctx:
        I, D = ctx.search_knn(q, 10, 512)
    for i in range(16):
        assert int(I[i, 0]) == int(planted[i])
        assert D[i, 0] < 1e-2
    _assert_knn_equal(x, q[:2], 1024, 10, 512, I[:2], D[:2])


def test_prepared_batch_reruns_and_kernel_switch():
    """A prepared batch (templates resident) gives the same answers on every run, under
    either contraction kernel."""
    x = _waveform(1 << 16, 31)
    m = 256
    q = _templates(x, m, np.random.default_rng(32), 4)
    reqs = [tb.Request(q[0], tb.MODE_KNN, k=8, merge_offset=128), tb.Request(q[1], tb.MODE_THRESHOLD, correlation=0.5),
            tb.Request(q[2], tb.MODE_KNN, k=3), tb.Request(q[3], tb.MODE_THRESHOLD, correlation=0.7, merge_offset=30)]
    with tb.Context(x) as ctx:
        b = ctx.batch(reqs)
        first = b.run()
        for kernel in [tb.KERNEL_FP32, tb.KERNEL_AUTO, tb.KERNEL_FP32]:
            ctx.set_kernel(kernel)
            again = b.run()
            for (p0, d0), (p1, d1) in zip(first, again):
                assert np.array_equal(p0, p1) and np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
        b.close()


def test_single_template_entry_points():
    """tm_scan_knn / tm_scan_threshold (one template, the worker seam's call): the same
    answers as the batch call; a caller's bound drops the answers above it."""
    x = _waveform(1 << 16, 91)
    m = 128
    q = _templates(x, m, np.random.default_rng(92), 2)
    with tb.Context(x) as ctx:
        (bp, bd), = ctx.scan_batch([tb.Request(q[0], tb.MODE_KNN, k=6, merge_offset=64)])
        p, d = ctx.scan_knn(q[0], 6, merge_offset=64)
        assert np.array_equal(p, bp) and np.array_equal(d.view(np.uint32), bd.view(np.uint32))
        p2, d2 = ctx.scan_knn(q[0], 6, merge_offset=64, bound=float(bd[2]))
        keep = bd <= bd[2]
        assert np.array_equal(p2, np.where(keep, bp, 0))
        assert np.array_equal(d2, np.where(keep, bd, np.finfo(np.float32).max))
        (tp_, td_), = ctx.scan_batch([tb.Request(q[1], tb.MODE_THRESHOLD, correlation=0.6, merge_offset=10)])
        p3, d3 = ctx.scan_threshold(q[1], 0.6, merge_offset=10)
        assert np.array_equal(p3, tp_) and np.array_equal(d3.view(np.uint32), td_.view(np.uint32))
