"""Randomised parity: seeded waveforms with the features the reference treats specially
(offsets, constant stretches, missing samples, loud and quiet stretches, repeated segments
whose windows tie), random batches of kNN and threshold requests of several lengths, an
optional window range, and every contraction branch (the planner's choice, row tiles,
column tiles, the FFT branch, the FP32 kernel): positions and distance bits equal the
oracle's in every case."""
import numpy as np
import pytest

import tremor_b200 as tb
from tests import oracle_bindings as ob

pytestmark = pytest.mark.gpu

BRANCHES = [('auto', tb.KERNEL_AUTO, tb.TILES_AUTO), ('rows', tb.KERNEL_AUTO, tb.TILES_ROWS),
            ('cols64', tb.KERNEL_AUTO, tb.TILES_COLS_64), ('fft', tb.KERNEL_AUTO, tb.TILES_FFT),
            ('fp32', tb.KERNEL_FP32, tb.TILES_AUTO)]


def _case(seed):
    from tremor_b200 import synth
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(3000, 70000))
    x = synth.ar2_waveform(n, rng) * np.float32(rng.uniform(0.1, 10.0)) + np.float32(rng.uniform(-50, 50))
    for _ in range(int(rng.integers(0, 3))):               # constant stretches
        a = int(rng.integers(0, n - 500))
        x[a:a + int(rng.integers(50, 500))] = np.float32(rng.uniform(-3, 3))
    for _ in range(int(rng.integers(0, 3))):               # loud / quiet stretches
        a = int(rng.integers(0, n - 2000))
        x[a:a + int(rng.integers(100, 2000))] *= np.float32(10.0 ** rng.uniform(-3, 3))
    seg = int(rng.integers(100, 600))                       # a repeated segment: tied windows
    a, b = int(rng.integers(0, n // 2 - seg)), int(rng.integers(n // 2, n - seg))
    x[b:b + seg] = x[a:a + seg]
    x[rng.integers(0, n, int(rng.integers(0, 40)))] = tb.MISSING_VALUE
    reqs = []
    for _ in range(int(rng.integers(1, 12))):
        m = int(8 * rng.integers(2, max(3, min(2048, n // 4) // 8)))
        kind = rng.integers(0, 3)
        if kind == 0:                                       # a window of the waveform (exact match)
            p = int(rng.integers(0, n - m))
            t = x[p:p + m].copy()
            t[t == tb.MISSING_VALUE] = 0.0
        elif kind == 1:
            t = synth.chirp_templates(1, m, rng)[0]
        else:
            t = rng.normal(size=m).astype(np.float32)
        if rng.random() < 0.05:
            t[:] = np.float32(2.0)                          # a constant template
        if rng.random() < 0.5:
            reqs.append(tb.Request(t, tb.MODE_KNN, k=int(rng.integers(1, 21)),
                                   merge_offset=int(rng.choice([0, int(rng.integers(1, m + 1))]))))
        else:
            reqs.append(tb.Request(t, tb.MODE_THRESHOLD, correlation=float(rng.uniform(-0.5, 0.99)),
                                   merge_offset=int(rng.choice([0, int(rng.integers(1, 64))]))))
    rng_range = None
    if rng.random() < 0.3:
        first = int(rng.integers(0, n // 3))
        rng_range = (first, int(rng.integers(n // 4, n)))
    return x, reqs, rng_range, BRANCHES[seed % len(BRANCHES)]


@pytest.mark.parametrize('seed', range(100))
def test_random_batches_match_oracle(seed):
    x, reqs, window_range, (name, kernel, tiles) = _case(seed)
    with tb.Context(x) as ctx:
        ctx.set_kernel(kernel)
        ctx.set_tiles(tiles)
        if window_range:
            ctx.set_window_range(*window_range)
        answers = ctx.scan_batch(reqs)
    first = window_range[0] if window_range else 0
    for r, (pos, dist) in zip(reqs, answers):
        m = len(r.template)
        if window_range:
            part = x[first:min(len(x), first + window_range[1] + m - 1)]
        else:
            part = x
        if len(part) < m:
            continue
        if r.mode == tb.MODE_KNN:
            I, D = ob.scan_knn(part, r.template[None, :], m, r.k, r.merge_offset)
            # padding is (0, FLT_MAX); a constant window answering an unfilled queue is
            # (position, FLT_MAX): relative position 0 is the one ambiguous case
            pad = (D[0] == np.float32(ob.FLT_MAX)) & (I[0] == 0)
            exp_pos = I[0] + first
            ok = (pos == exp_pos) | (pad & (pos == 0))
            assert np.all(ok), (name, seed, m, r.k, r.merge_offset)
            assert np.array_equal(dist.view(np.uint32), D[0].view(np.uint32)), (name, seed, m)
        else:
            _, p, d = ob.scan_threshold(part, r.template[None, :], m, r.correlation, r.merge_offset)
            assert np.array_equal(pos, p + first), (name, seed, m, r.correlation, r.merge_offset)
            assert np.array_equal(dist.view(np.uint32), d.view(np.uint32)), (name, seed, m)
