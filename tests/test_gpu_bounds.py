"""The per-result error bound of each contraction kernel holds.

For every (template, window) pair, |d - reference FP32 distance| <= e, where d is the
contraction kernel's distance (FP32 CUDA cores, or split-BF16 tensor cores) and e the
bound its fused epilogue uses to decide which windows are re-scored exactly. This is
what makes the answer sets exact; the test also reports how tight the bound is."""
import numpy as np
import pytest

import tremor_b200 as tb
from tests.test_gpu_parity import _templates, _waveform

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('kernel', [tb.KERNEL_FP32, tb.KERNEL_AUTO])
@pytest.mark.parametrize('m', [48, 100, 256, 1000, 4096])
def test_bound_holds_everywhere(kernel, m):
    x = _waveform(1 << 16, 40 + m)
    q = _templates(x, m, np.random.default_rng(m + 41), 6)
    with tb.Context(x) as ctx:
        ctx.set_kernel(kernel)
        d, e, exact = ctx.bound_diagnostics(q)
    ok = np.isfinite(d) & (exact < np.float32(3.0e38))
    assert ok.sum() > 0.9 * ok.size * 0.5
    err = np.abs(d[ok].astype(np.float64) - exact[ok].astype(np.float64))
    assert np.all(err <= e[ok]), (m, float(np.max(err / e[ok])))
    ratio = float(np.max(err / e[ok]))
    print(f'kernel={kernel} m={m}: max |d-exact|/e = {ratio:.3g}, median e/(2m) = {np.median(e[ok]) / (2 * m):.3g}')


@pytest.mark.parametrize('tiles', [tb.TILES_COLS_128, tb.TILES_COLS_64, tb.TILES_COLS_32, tb.TILES_FFT])
@pytest.mark.parametrize('m', [48, 100, 1000, 4096])
def test_bound_holds_window_major(tiles, m):
    """The same for the window-major kernel (templates in column tiles, window statistics
    from the prefix sums with their own error term). Its waveform keeps the loud stretch
    moderate: after a 1e5-fold one the prefix sums leave most later windows to the exact
    re-scoring (statistics flagged untrustworthy), which would leave little to check."""
    from tremor_b200 import synth
    rng = np.random.default_rng(60 + m)
    x = synth.ar2_waveform(1 << 16, rng) + np.float32(3.0)
    x[1000:4000] = 2.0
    x[20000:24000] *= np.float32(30.0)
    x[24000:30000] *= np.float32(0.05)
    x[rng.integers(0, len(x), 50)] = tb.MISSING_VALUE
    q = _templates(x, m, np.random.default_rng(m + 61), 6)
    with tb.Context(x) as ctx:
        ctx.set_tiles(tiles)
        d, e, exact = ctx.bound_diagnostics(q)
    ok = np.isfinite(d) & (exact < np.float32(3.0e38))
    assert ok.sum() > 0.9 * ok.size * 0.5
    err = np.abs(d[ok].astype(np.float64) - exact[ok].astype(np.float64))
    assert np.all(err <= e[ok]), (m, float(np.max(err / e[ok])))


@pytest.mark.parametrize('tiles', [tb.TILES_COLS_64, tb.TILES_FFT])
@pytest.mark.parametrize('m', [100, 4096, 16384])
def test_bound_holds_across_prefix_blocks(m, tiles):
    """The window-major kernel's bound with block-local prefix sums, on a record with level
    steps at the block boundaries and a 1e5-fold loud stretch in block 0: the bound holds,
    and windows two blocks after the loud stretch keep trustworthy statistics (the prefix
    sums' error bound is local)."""
    from tests.test_gpu_batching import _block_waveform
    x = _block_waveform(70 + m)
    q = _templates(x, m, np.random.default_rng(m + 71), 4)
    with tb.Context(x) as ctx:
        ctx.set_tiles(tiles)
        d, e, exact = ctx.bound_diagnostics(q)
    ok = np.isfinite(d) & (exact < np.float32(3.0e38))
    err = np.abs(d[ok].astype(np.float64) - exact[ok].astype(np.float64))
    assert np.all(err <= e[ok]), (m, float(np.max(err / e[ok])))
    later = ok[:, 2 * 65536:2 * 65536 + 40000]
    assert later.mean() > 0.95, float(later.mean())
