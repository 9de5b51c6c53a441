"""tm_result_fp64 against an independent FP64 recomputation.

Every answer of a batch carries, through tm_result_fp64, the squared z-normalised distance
of its (template, window) recomputed in FP64 on the device from the raw samples. Here the
same quantity is computed again in NumPy (float64, missing samples -100000 counted as 0 as
SkipSequential.cpp:157-190 does, a window or template with std <= 1e-12 treated as
constant) for every answer of the golden fixtures and of a record with constant stretches:

* answers with a finite FP32 distance: the device's FP64 value within 1e-12 relative
  (plus 1e-9 absolute, for distances near 0) of NumPy's;
* padding (kNN slots the exclusion zone leaves empty, distance FLT_MAX, as the 'sparse'
  fixture has): +inf;
* the returned FP32 distance within the FP32 error model of FP64 wherever FP64 is finite:
  |D - D64| <= 1e-4 D64 + 2^-20 sqrt(m D64) + m 2^-44 (1e-4 relative away from 0; exact
  copies of a template, distance near 0, are held to the absolute terms).
"""
import numpy as np
import pytest

import tremor_b200 as tb
from tests import oracle_bindings as ob

pytestmark = pytest.mark.gpu

MISSING = -100000.0


def _znorm64(v):
    v = np.where(v == MISSING, 0.0, v.astype(np.float64))
    mu = v.mean()
    sd = np.sqrt(np.mean((v - mu) ** 2))
    return None if sd <= 1e-12 else (v - mu) / sd


def _numpy_fp64(x, template, positions):
    m = len(template)
    q = _znorm64(template)
    if q is None:
        q = np.zeros(m)
    out = np.empty(len(positions))
    for j, p in enumerate(positions):
        w = _znorm64(x[int(p):int(p) + m])
        out[j] = np.inf if w is None else np.sum((q - w) ** 2)
    return out


def _check(x, requests, answers, what):
    padded = 0
    for r, (pos, dist, d64) in zip(requests, answers):
        pad = dist >= ob.FLT_MAX
        padded += int(pad.sum())
        assert np.all(np.isposinf(d64[pad])), f'{what}: padding must report +inf'
        ref = _numpy_fp64(x, r.template, pos[~pad])
        got = d64[~pad]
        assert np.all(np.isfinite(ref)), f'{what}: an answer on a constant window'
        assert np.all(np.abs(got - ref) <= 1e-12 * ref + 1e-9), (what, np.max(np.abs(got - ref)))
        # the FP32 error model of the reference's distance (exact copies have distances near 0,
        # where its absolute error of a few ulps of the per-sample terms dominates)
        m = len(r.template)
        err = np.abs(dist[~pad].astype(np.float64) - got)
        assert np.all(err <= 1e-4 * got + 2.0 ** -20 * np.sqrt(m * got) + m * 2.0 ** -44), (what, err.max())
    return padded


@pytest.mark.parametrize('name', ob.golden_cases())
def test_golden_answers_fp64(name):
    meta, x, q = ob.load_golden(name)
    padded = 0
    with tb.Context(x) as ctx:
        for merge in meta['merges']:
            reqs = [tb.Request(t, tb.MODE_KNN, k=meta['k'], merge_offset=merge) for t in q]
            reqs += [tb.Request(t, tb.MODE_THRESHOLD, correlation=meta['threshold'], merge_offset=merge) for t in q]
            answers = ctx.scan_batch(reqs, fp64=True)
            padded += _check(x, reqs, answers, f'{name} merge {merge}')
    if name == 'sparse':
        assert padded > 0, 'the sparse fixture should leave kNN slots empty'


def test_constant_stretches_fp64():
    """A record with long constant stretches (their windows are never answers) and a
    quiet stretch (std just above the constant limit): kNN with k larger than the windows
    outside the exclusion zone, so that padding appears, and a low threshold."""
    rng = np.random.default_rng(17)
    n, m = 1 << 15, 256
    x = rng.normal(size=n).astype(np.float32)
    x[2000:9000] = 3.0
    x[12000:12800] = (1.0 + 1e-4 * rng.normal(size=800)).astype(np.float32)
    x[20000:20040] = MISSING
    q = [x[15000:15000 + m].copy(), rng.normal(size=m).astype(np.float32)]
    reqs = [tb.Request(t, tb.MODE_KNN, k=100, merge_offset=m * 8) for t in q]
    reqs += [tb.Request(t, tb.MODE_THRESHOLD, correlation=0.2, merge_offset=0) for t in q]
    with tb.Context(x) as ctx:
        answers = ctx.scan_batch(reqs, fp64=True)
    assert _check(x, reqs, answers, 'constant stretches') > 0
    assert answers[0][0][0] == 15000 and answers[0][2][0] < 1e-6
