"""Tile shapes of the tensor-core contraction: the autotuner's measured model, its use by
the planner (TM_TILES_AUTO), and that a forced shape runs the kernel it names."""
import numpy as np
import pytest

import tremor_b200 as tb
from tests.test_gpu_batching import _check, _requests, _waveform

pytestmark = pytest.mark.gpu


def test_autotune_model():
    x = _waveform(1 << 16, 31)
    with tb.Context(x) as ctx:
        table, fft_ms, fft_long_ms = ctx.autotune()
        assert table.shape == (2, 4, 4) and np.all(np.isfinite(table)) and np.all(table > 0)
        assert np.isfinite(fft_ms) and fft_ms > 0 and np.isfinite(fft_long_ms) and fft_long_ms > 0
        # more samples per window cost more on every shape; long templates favour wide tiles
        assert np.all(np.diff(table[:, :, 1:], axis=2) > 0)
        assert np.all(table[:, 0, 3] < table[:, 3, 3])
        ctx.set_tile_model(table, fft_ms, fft_long_ms)
        with pytest.raises(tb.TremorError):
            ctx.set_tile_model(np.zeros(32))


@pytest.mark.parametrize('tiles,kernel', [(tb.TILES_ROWS, 'k_scan_umma'), (tb.TILES_COLS_64, 'k_scan_wm')])
def test_forced_shape_runs_its_kernel(tiles, kernel):
    x = _waveform(1 << 16, 32)
    rng = np.random.default_rng(33)
    reqs = _requests(x, rng, [64, 100, 200, 64, 512])
    with tb.Context(x) as ctx:
        ctx.set_tiles(tiles)
        ctx.profile_enable(True)
        answers = ctx.scan_batch(reqs)
        name = ctx.profile_read()[0]
    assert name == kernel
    _check(x, reqs, answers)


def test_planner_follows_the_model():
    """AUTO picks the shape of least modelled time: row tiles under a model where they are
    cheapest, 32-template column tiles under one where those are; the answers do not
    depend on the choice."""
    x = _waveform(1 << 16, 34)
    rng = np.random.default_rng(35)
    reqs = _requests(x, rng, [64, 100, 200, 64, 512])
    cheap_rows = np.full((2, 4, 4), 100.0)
    cheap_rows[:, 0, :] = 1.0
    cheap_cols = np.full((2, 4, 4), 100.0)
    cheap_cols[:, 3, :] = 1.0
    with tb.Context(x) as ctx:
        ctx.profile_enable(True)
        ctx.set_tile_model(cheap_rows)
        base = ctx.scan_batch(reqs)
        assert ctx.profile_read()[0] == 'k_scan_umma'
        ctx.set_tile_model(cheap_cols)
        again = ctx.scan_batch(reqs)
        assert ctx.profile_read()[0] == 'k_scan_wm'
    for (p0, d0), (p1, d1) in zip(base, again):
        assert np.array_equal(p0, p1) and np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
    _check(x, reqs, base)


def test_planner_picks_fft_for_a_long_template():
    """One long template: a 128-row tile would be mostly padding, the FFT branch's cost does
    not grow with the length, so AUTO (default model) takes the FFT branch; the answers
    equal the oracle's and the row tiles'."""
    x = _waveform(1 << 17, 36)
    t = x[40000:40000 + 8192].copy()
    t[t == tb.MISSING_VALUE] = 0.0
    reqs = [tb.Request(t, tb.MODE_KNN, k=4, merge_offset=4096)]
    with tb.Context(x) as ctx:
        ctx.profile_enable(True)
        auto = ctx.scan_batch(reqs)
        assert ctx.profile_read()[0] == 'fft'
        ctx.set_tiles(tb.TILES_ROWS)
        rows = ctx.scan_batch(reqs)
        assert ctx.profile_read()[0] == 'k_scan_umma'
    assert np.array_equal(auto[0][0], rows[0][0])
    assert np.array_equal(auto[0][1].view(np.uint32), rows[0][1].view(np.uint32))
    _check(x, reqs, auto)


def test_planner_splits_long_tail_to_fft():
    """A batch with a few very long templates and many short ones: under the default model
    the longest go to the FFT branch and the rest to row tiles (two groups, both kernels
    run); the answers equal the oracle's and those of row tiles alone."""
    x = _waveform(1 << 17, 37)
    rng = np.random.default_rng(38)
    reqs = _requests(x, rng, [16384, 12000] + [int(v) for v in rng.choice([64, 96, 128, 200], size=130)])
    with tb.Context(x) as ctx:
        ctx.profile_enable(True)
        ctx.profile_phases()
        auto = ctx.scan_batch(reqs)
        ctx.profile_read()
        ctx.set_tiles(tb.TILES_ROWS)
        rows = ctx.scan_batch(reqs)
    for (p0, d0), (p1, d1) in zip(auto, rows):
        assert np.array_equal(p0, p1) and np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
    _check(x, reqs, auto)
