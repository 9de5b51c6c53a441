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
