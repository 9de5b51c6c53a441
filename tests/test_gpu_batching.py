"""Batches of templates of different lengths (one mixed-length contraction group whose
window statistics come from the resident FP64 prefix sums) give exactly the reference's
answers: positions and FP32 distance bits equal to the oracle's, for kNN and threshold
requests mixed in one batch, on waveforms with missing samples, long constant stretches,
a loud stretch followed by a quiet one (prefix-sum cancellation), and a large offset."""
import numpy as np
import pytest

import tremor_b200 as tb
from tests import oracle_bindings as ob

pytestmark = pytest.mark.gpu

# every branch of the mixed-length contraction: 128-template row tiles (k_scan_umma),
# column tiles of 128 / 64 / 32 templates (k_scan_wm), the FP64 FFT branch (tm_fftk.cu)
TILES = [tb.TILES_ROWS, tb.TILES_COLS_128, tb.TILES_COLS_64, tb.TILES_COLS_32, tb.TILES_FFT]


def _waveform(n, seed, offset=0.0):
    from tremor_b200 import synth
    rng = np.random.default_rng(seed)
    x = synth.ar2_waveform(n, rng) + np.float32(offset)
    x[3000:9000] = np.float32(offset)               # long constant stretch
    x[30000:34000] *= np.float32(1e5)               # loud ...
    x[34000:40000] *= np.float32(1e-4)              # ... then quiet
    x[rng.integers(0, n, 60)] = tb.MISSING_VALUE    # scattered missing samples
    x[60000:60200] = tb.MISSING_VALUE               # a gap
    return x


def _requests(x, rng, lengths):
    from tremor_b200 import synth
    reqs = []
    for i, m in enumerate(lengths):
        if i % 3 == 0:
            p = int(rng.integers(0, len(x) - m))
            t = x[p:p + m].copy()
            t[t == tb.MISSING_VALUE] = 0.0
        else:
            t = synth.chirp_templates(1, m, rng)[0]
        if i % 2 == 0:
            reqs.append(tb.Request(t, tb.MODE_KNN, k=int(rng.choice([1, 5, 20])),
                                   merge_offset=int(rng.choice([0, m // 2]))))
        else:
            reqs.append(tb.Request(t, tb.MODE_THRESHOLD, correlation=float(rng.choice([0.3, 0.6, 0.85])),
                                   merge_offset=int(rng.choice([0, 10]))))
    return reqs


def _check(x, reqs, answers):
    for r, (pos, dist) in zip(reqs, answers):
        m = len(r.template)
        if r.mode == tb.MODE_KNN:
            I, D = ob.scan_knn(x, r.template[None, :], m, r.k, r.merge_offset)
            assert np.array_equal(pos, I[0]), (m, r.k, r.merge_offset)
            assert np.array_equal(dist.view(np.uint32), D[0].view(np.uint32)), (m, r.k)
        else:
            qid, p, d = ob.scan_threshold(x, r.template[None, :], m, r.correlation, r.merge_offset)
            assert np.array_equal(pos, p), (m, r.correlation, r.merge_offset)
            assert np.array_equal(dist.view(np.uint32), d.view(np.uint32))


@pytest.mark.parametrize('tiles', TILES)
@pytest.mark.parametrize('offset', [0.0, 5000.0])
def test_mixed_lengths_match_oracle(offset, tiles):
    x = _waveform(1 << 17, 5 + int(offset), offset)
    rng = np.random.default_rng(6)
    lengths = [int(v) for v in rng.choice([40, 64, 100, 128, 200, 333, 512, 1000, 2048], size=18)]
    reqs = _requests(x, rng, lengths)
    with tb.Context(x) as ctx:
        ctx.set_tiles(tiles)
        answers = ctx.scan_batch(reqs)
    _check(x, reqs, answers)


@pytest.mark.parametrize('tiles', TILES)
def test_mixed_lengths_window_range(tiles):
    x = _waveform(1 << 16, 8)
    rng = np.random.default_rng(9)
    reqs = _requests(x, rng, [64, 96, 150, 300, 64, 500])
    first, count = 7000, 40000
    with tb.Context(x) as ctx:
        ctx.set_tiles(tiles)
        ctx.set_window_range(first, count)
        answers = ctx.scan_batch(reqs)
    for r, (pos, dist) in zip(reqs, answers):
        m = len(r.template)
        part = x[first:min(len(x), first + count + m - 1)]
        if r.mode == tb.MODE_KNN:
            I, D = ob.scan_knn(part, r.template[None, :], m, r.k, r.merge_offset)
            assert np.array_equal(pos, np.where(D[0] < ob.FLT_MAX, I[0] + first, 0))
            assert np.array_equal(dist.view(np.uint32), D[0].view(np.uint32))
        else:
            qid, p, d = ob.scan_threshold(part, r.template[None, :], m, r.correlation, r.merge_offset)
            assert np.array_equal(pos, p + first)
            assert np.array_equal(dist.view(np.uint32), d.view(np.uint32))


@pytest.mark.parametrize('tiles', TILES)
def test_mixed_lengths_sparse_unbounded(tiles):
    """So few windows that no kNN bound exists: constant windows (distance FLT_MAX) fill
    the answers in position order, as the reference's unfilled queue makes them do."""
    rng = np.random.default_rng(10)
    x = rng.normal(size=600).astype(np.float32)
    x[100:260] = 3.0
    reqs = [tb.Request(x[20:84].copy(), tb.MODE_KNN, k=12, merge_offset=40),
            tb.Request(rng.normal(size=100).astype(np.float32), tb.MODE_KNN, k=9, merge_offset=30),
            tb.Request(rng.normal(size=48).astype(np.float32), tb.MODE_THRESHOLD, correlation=-0.2)]
    with tb.Context(x) as ctx:
        ctx.set_tiles(tiles)
        answers = ctx.scan_batch(reqs)
    _check(x, reqs, answers)


@pytest.mark.parametrize('tiles', [tb.TILES_ROWS, tb.TILES_COLS_64, tb.TILES_FFT])
def test_constant_stretch_does_not_flood_candidates(tiles):
    """Windows inside a long constant stretch are recognised from the constant-run lengths,
    not handed one by one to the exact re-scoring."""
    from tremor_b200 import synth
    rng = np.random.default_rng(12)
    x = synth.ar2_waveform(1 << 18, rng)
    x[10000:200000] = 0.0
    reqs = [tb.Request(synth.chirp_templates(1, m, rng)[0], tb.MODE_THRESHOLD, correlation=0.9)
            for m in [64, 128, 256, 512]]
    with tb.Context(x) as ctx:
        ctx.set_tiles(tiles)
        ctx.scan_batch(reqs)
        assert ctx.last_candidates() < 5000


@pytest.mark.parametrize('tiles', TILES)
def test_mixed_lengths_last_windows(tiles):
    """A template planted in the last window of the waveform (or a few samples before it)
    is found with its exact distance while templates of other lengths share its tiles
    (the window-end prefix sums at the end of the record)."""
    rng = np.random.default_rng(13)
    n = 50000
    lengths = [100, 333, 64, 1000]
    temps = [rng.normal(size=m).astype(np.float32) for m in lengths]
    for k, m in enumerate(lengths):
        x = rng.normal(size=n).astype(np.float32)
        end = n - 7 * k  # the last window, or a few before it
        x[end - m:end] = temps[k] * np.float32(2.0) + np.float32(1.0)
        reqs = []
        for t in temps:
            reqs.append(tb.Request(t, tb.MODE_KNN, k=1))
            reqs.append(tb.Request(t, tb.MODE_THRESHOLD, correlation=0.99))
        with tb.Context(x) as ctx:
            ctx.set_tiles(tiles)
            answers = ctx.scan_batch(reqs)
        assert int(answers[2 * k][0][0]) == end - m
        assert end - m in set(int(p) for p in answers[2 * k + 1][0])
        _check(x, reqs, answers)


def test_results_outlive_later_searches():
    """A result keeps its answers while later searches of the same context run and are
    freed (the answers live in pinned blocks that the result holds)."""
    import ctypes
    x = _waveform(1 << 16, 14)
    rng = np.random.default_rng(15)
    reqs_a = _requests(x, rng, [64, 100, 200, 64])
    reqs_b = _requests(x, rng, [128, 300, 96, 512, 40])
    with tb.Context(x) as ctx:
        ref_a, ref_b = ctx.scan_batch(reqs_a), ctx.scan_batch(reqs_b)
        held = []
        for reqs in (reqs_a, reqs_b, reqs_a):
            res = ctypes.c_void_p()
            ctx._check(ctx._lib.tm_scan_batch(ctx._h, ctx._requests(reqs), len(reqs), ctypes.byref(res)))
            held.append(res)
        ctx.scan_batch(reqs_b)  # one more search, its result freed at once
        got = [ctx._take(r, n) for r, n in zip(held, (len(reqs_a), len(reqs_b), len(reqs_a)))]
    for answers, ref in zip(got, (ref_a, ref_b, ref_a)):
        for (p, d), (rp, rd) in zip(answers, ref):
            assert np.array_equal(p, rp) and np.array_equal(d.view(np.uint32), rd.view(np.uint32))
    _check(x, reqs_a, ref_a)
    _check(x, reqs_b, ref_b)


def test_large_k_selected_on_host():
    """k above the device selection's limit (1024 kept windows per template) takes the
    host selection over the sorted run; its answers match the oracle too, next to a
    request that the device selects."""
    x = _waveform(1 << 15, 16)
    rng = np.random.default_rng(17)
    reqs = [tb.Request(x[500:564].copy(), tb.MODE_KNN, k=1500, merge_offset=3),
            tb.Request(x[900:1028].copy(), tb.MODE_KNN, k=20, merge_offset=64),
            tb.Request(rng.normal(size=96).astype(np.float32), tb.MODE_THRESHOLD, correlation=0.5)]
    with tb.Context(x) as ctx:
        answers = ctx.scan_batch(reqs)
    _check(x, reqs, answers)


def _block_waveform(seed):
    """Three prefix blocks (65536 samples) and a bit: a level step at each block boundary,
    a 1e5-fold loud stretch in block 0, missing samples; many windows cross a boundary."""
    from tremor_b200 import synth
    rng = np.random.default_rng(seed)
    n = 3 * 65536 + 5000
    x = synth.ar2_waveform(n, rng)
    x[65536:131072] += np.float32(1000.0)
    x[131072:] -= np.float32(500.0)
    x[20000:24000] *= np.float32(1e5)
    x[rng.integers(0, n, 40)] = tb.MISSING_VALUE
    return x


@pytest.mark.parametrize('tiles', [tb.TILES_ROWS, tb.TILES_COLS_64, tb.TILES_FFT])
def test_prefix_blocks_and_loud_event(tiles):
    """Statistics from block-local prefix sums across block boundaries with level steps, and
    after a loud event: answers equal the oracle's."""
    x = _block_waveform(41)
    rng = np.random.default_rng(42)
    reqs = []
    for i, m in enumerate([16384, 8000, 4096, 1000, 333, 64, 16384, 2048]):
        p = int(rng.integers(60000, 140000))
        t = x[p:p + m].copy()
        t[t == tb.MISSING_VALUE] = 0.0
        reqs.append(tb.Request(t, tb.MODE_KNN, k=3, merge_offset=m // 2) if i % 2 == 0
                    else tb.Request(t, tb.MODE_THRESHOLD, correlation=0.7))
    with tb.Context(x) as ctx:
        ctx.set_tiles(tiles)
        answers = ctx.scan_batch(reqs)
    _check(x, reqs, answers)


@pytest.mark.parametrize('tiles', [tb.TILES_ROWS, tb.TILES_COLS_128])
def test_many_distinct_lengths_per_tile(tiles):
    """Row tiles hold 128 templates whatever their lengths: 160 templates, the first 130 of
    distinct lengths (every epilogue warp of the first tile sees 32 lengths, its table's
    maximum), the rest sharing lengths across warp boundaries; answers equal the oracle's."""
    x = _waveform(1 << 15, 77)
    x = x[:20000].copy()
    rng = np.random.default_rng(78)
    lengths = [16 + 4 * i for i in range(130)] + [int(v) for v in rng.choice([40, 41, 200, 517], size=30)]
    rng.shuffle(lengths)
    reqs = _requests(x, rng, lengths)
    with tb.Context(x) as ctx:
        ctx.set_tiles(tiles)
        answers = ctx.scan_batch(reqs)
    _check(x, reqs, answers)


def test_batches_created_and_destroyed_reuse_memory():
    """Batches created, run and destroyed one after another take their device buffers
    from the memory pool and give them back: the answers stay identical and the device's
    free memory does not shrink from cycle to cycle."""
    import torch
    x = _waveform(1 << 17, 91)
    rng = np.random.default_rng(92)
    reqs = _requests(x, rng, [64, 200, 1000, 64, 333, 2048, 4096])
    free, first = [], None
    with tb.Context(x) as ctx:
        for _ in range(20):
            b = ctx.batch(reqs)
            out = b.run()
            b.close()
            if first is None:
                first = out
            for (p0, d0), (p1, d1) in zip(first, out):
                assert np.array_equal(p0, p1) and np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
    assert free[-1] >= free[1] - (16 << 20), (free[1], free[-1])
    _check(x, reqs, first)
