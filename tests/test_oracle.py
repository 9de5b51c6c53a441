"""The oracle (oracle/tm_oracle.c) pinned against the reference.

1. Golden answers: for every committed fixture, the oracle's kNN and threshold
   answers, printed as the reference's CSV writers print them, equal the rows the
   reference's own SkipSequentialScan produced (tests/golden/make_golden.py).
2. Bit-level pin (where oracle/_ref was built from the reference sources): the
   oracle's z-normalisation, block order, window statistics and early-abandoning
   distance are bit-identical to the reference's compiled ones on random inputs.
3. The FP64 Pearson oracle of experiments/validate_search.py:80-148 accepts the
   oracle's answers on the validate case (correlations within 2e-4, exact kNN sets
   with and without exclusion zone, threshold set equality).
"""
import os
import tempfile

import numpy as np
import pytest

from tests import oracle_bindings as ob


@pytest.mark.parametrize('name', ob.golden_cases())
def test_oracle_matches_golden_knn(name):
    meta, x, q = ob.load_golden(name)
    for merge in meta['merges']:
        I, D = ob.scan_knn(x, q, meta['m'], meta['k'], merge)
        assert ob.knn_rows(I, D, meta['m']) == meta['knn'][str(merge)], (name, merge)


@pytest.mark.parametrize('name', ob.golden_cases())
def test_oracle_matches_golden_threshold(name):
    meta, x, q = ob.load_golden(name)
    for merge in meta['merges']:
        qid, pos, dist = ob.scan_threshold(x, q, meta['m'], meta['threshold'], merge)
        assert ob.threshold_rows(qid, pos, dist, meta['m']) == meta['threshold_hits'][str(merge)], (name, merge)


ref = ob.reference()


@pytest.mark.skipif(ref is None, reason='reference build (oracle/_ref) not present')
def test_oracle_bit_identical_to_reference_kernels():
    lib = ob.oracle()
    P = ob.P
    rng = np.random.default_rng(11)
    checks = 0
    with tempfile.TemporaryDirectory() as tmp:
        wf = os.path.join(tmp, 'w.bin')
        for trial in range(40):
            m = int(rng.choice([32, 48, 64, 72, 100, 256, 1000]))
            q = (rng.normal(size=m) * rng.uniform(0.01, 100)).astype(np.float32)
            q1, q2 = q.copy(), q.copy()
            lib.tmo_znormalize(P(q1), m)
            ref.tmref_znormalize(P(q2), m)
            assert np.array_equal(q1.view(np.uint32), q2.view(np.uint32))
            o1 = np.zeros(m // 32 + 1, np.int32)
            o2 = np.zeros(m // 32 + 1, np.int32)
            lib.tmo_block_order(P(q1), m, P(o1))
            ref.tmref_block_order(P(q1), m, P(o2))
            assert np.array_equal(o1, o2)
            n = 3000
            x = (rng.normal(size=n) * rng.uniform(0.01, 1e4) + rng.uniform(-10, 10)).astype(np.float32)
            x[rng.integers(0, n, 15)] = ob.np.float32(-100000.0)
            x[500:500 + m + 5] = 2.5  # constant windows
            x[1200:1300] *= np.float32(1e-4)
            x.tofile(wf)
            W = n - m + 1
            mo, so, mr, sr = (np.zeros(W, np.float32) for _ in range(4))
            lib.tmo_window_stats(P(x), W, m, P(mo), P(so))
            assert ref.tmref_sss_stats(wf.encode(), n, m, 1, P(mr), P(sr)) == 0
            assert np.array_equal(mo.view(np.uint32), mr.view(np.uint32))
            assert np.array_equal(so.view(np.uint32), sr.view(np.uint32))
            bv = ob.ctypes.c_int(0)
            for j in rng.integers(0, W, 40):
                bound = float(rng.choice([ob.FLT_MAX, 10.0 * m, 1.0 * m]))
                args = (P(q1), P(x), int(j), m, float(mr[j]), float(sr[j]), bound, P(o1), ob.ctypes.byref(bv))
                d1, d2 = lib.tmo_l2_dist(*args), ref.tmref_l2_dist(*args)
                assert np.float32(d1).view(np.uint32) == np.float32(d2).view(np.uint32)
                checks += 1
    assert checks == 1600


def _fp64_correlations(x, queries, m):
    """experiments/validate_search.py:80-86 (FP64 Pearson oracle)."""
    windows = np.lib.stride_tricks.sliding_window_view(x.astype('float64'), m)
    with np.errstate(invalid='ignore', divide='ignore'):
        zn = (windows - windows.mean(axis=1)[:, None]) / windows.std(axis=1)[:, None]
    qn = queries.astype('float64') - queries.mean(axis=1, dtype='float64')[:, None]
    qn /= qn.std(axis=1)[:, None]
    corr = qn @ zn.T / m
    corr[:, windows.std(axis=1) <= 1e-12] = -np.inf
    return corr


def _knn_with_exclusion(correlations, k, merge):
    """experiments/validate_search.py:20-30."""
    order = sorted(range(len(correlations)), key=lambda p: (-correlations[p], p))
    kept = []
    for p in order:
        if len(kept) == k or correlations[p] == -np.inf:
            break
        if all(abs(p - q) >= merge for q in kept):
            kept.append(p)
    return kept


def test_oracle_passes_validate_search_checks():
    meta, x, q = ob.load_golden('validate')
    m, k, n = meta['m'], meta['k'], len(x)
    corr = _fp64_correlations(x, q, m)
    for merge in meta['merges']:
        I, D = ob.scan_knn(x, q, m, k, merge)
        for qi in range(len(q)):
            actual = [int(p) for p in I[qi]]
            cc = [ob.ed_to_cc(d, m) for d in D[qi]]
            assert np.allclose(cc, corr[qi, actual], atol=2e-4)
            expected = (np.argsort(-corr[qi], kind='stable')[:k].tolist() if merge == 0
                        else _knn_with_exclusion(corr[qi], k, merge))
            assert actual == expected
        qid, pos, dist = ob.scan_threshold(x, q, m, meta['threshold'], merge)
        for qi in range(len(q)):
            actual = set(int(p) for p in pos[qid == qi])
            expected, next_allowed = set(), 0  # one partition (validate_search.py:136-148)
            for p in np.flatnonzero(corr[qi, :n - m + 1] >= meta['threshold']):
                if p >= next_allowed:
                    expected.add(int(p))
                    next_allowed = p + merge + 1
            assert actual == expected
            cc = [ob.ed_to_cc(d, m) for d in dist[qid == qi]]
            assert np.allclose(cc, corr[qi, sorted(actual)], atol=2e-4)


def test_mass_v3_restatement_matches_fp64_oracle():
    """oracle/mass_v3.py (DMASS_V3.c:798-996 with pocketfft for FFTW) gives the FP64
    distances of validate_search's oracle to 1e-9 relative, and its kNN answers are the
    FP64 expectations of validate_search.py:128-135."""
    import sys
    sys.path.insert(0, str(ob.ROOT / 'oracle'))
    from mass_v3 import MassV3
    meta, x, q = ob.load_golden('validate')
    m, k = meta['m'], meta['k']
    corr = _fp64_correlations(x, q, m)
    mass = MassV3(x, m, workers=2)
    for qi in range(len(q)):
        d = mass.distances(q[qi])
        ok = np.isfinite(corr[qi]) & (corr[qi] > -np.inf)
        expect = 2 * m * (1 - corr[qi][ok])
        assert np.allclose(d[ok], expect, rtol=1e-9, atol=1e-7 * m)
        order = sorted(range(len(d)), key=lambda p: (d[p], p))[:k]
        assert order == np.argsort(-corr[qi], kind='stable')[:k].tolist()


@pytest.mark.skipif(ref is None, reason='reference build (oracle/_ref) not present')
def test_fast_window_stats_bit_identical_to_reference_build():
    """tmo_window_stats_fast (the statistics of the full-size parity checks) equals, bit for
    bit, what the reference's SkipSequentialScan::build computes (SkipSequential.cpp:157-190),
    with missing samples, constant stretches and loud stretches in the record."""
    rng = np.random.default_rng(23)
    n = 1 << 18
    x = (rng.normal(size=n) * 3.0 + 7.0).astype(np.float32)
    x[1000:1040] = np.float32(-100000.0)
    x[5000:9000] = 2.5
    x[20000:20500] *= np.float32(1e5)
    x[70001] = np.float32(-100000.0)
    with tempfile.TemporaryDirectory() as tmp:
        wf = os.path.join(tmp, 'w.bin')
        x.tofile(wf)
        for m in (16, 100, 256, 1000, 4096):
            W = n - m + 1
            rm = np.zeros(W, np.float32)
            rs = np.zeros(W, np.float32)
            assert ref.tmref_sss_stats(wf.encode(), n, m, 4, ob.P(rm), ob.P(rs)) == 0
            fm, fs = ob.window_stats_fast(x, m)
            assert np.array_equal(rm.view(np.uint32), fm.view(np.uint32)), m
            assert np.array_equal(rs.view(np.uint32), fs.view(np.uint32)), m


@pytest.mark.skipif(ref is None, reason='reference build (oracle/_ref) not present')
@pytest.mark.parametrize('name', ['validate', 'chirp'])
def test_reference_scan_from_stats_equals_golden(name):
    """The reference's own scan over a record in memory with the oracle's statistics
    (ReferenceScan, the full-size parity checks' reference) prints exactly the golden
    rows that the reference's build() + search produced."""
    meta, x, q = ob.load_golden(name)
    m = meta['m']
    for merge in meta['merges']:
        with ob.ReferenceScan(x, m, merge_offset=merge, threads=4) as rs:
            knn = rs.knn(q, meta['k'])
            rows = [[str(i), str(j + 1), str(int(p)), c] for i, (pos, cc) in enumerate(knn)
                    for j, (p, c) in enumerate(zip(pos, cc))]
            assert rows == meta['knn'][str(merge)], (name, merge)
            thr = rs.threshold(q, meta['threshold'])
            rows = [[str(i), str(c), str(int(p)), cc] for i, (pos, ccs) in enumerate(thr)
                    for c, (p, cc) in enumerate(zip(pos, ccs))]
            assert rows == meta['threshold_hits'][str(merge)], (name, merge)
            # the reference's distance bits at its own answers equal the oracle's
            Io, Do = ob.scan_knn(x, q, m, meta['k'], merge)
            for i in range(len(q)):
                ok = Do[i] < ob.FLT_MAX
                d = rs.distances(q[i], Io[i][ok])
                assert np.array_equal(d.view(np.uint32), Do[i][ok].view(np.uint32)), (name, merge, i)
