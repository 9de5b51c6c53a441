"""ctypes bindings of the CPU oracle (oracle/tm_oracle.c) and of the reference's own
scan build (oracle/_ref/libtremor_ref.so, present only where it was built).

Test infrastructure: used by tests/ and bench.py's CPU-baseline leg only."""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / 'tests' / 'golden'
FLT_MAX = float(np.finfo(np.float32).max)

_vp = ctypes.c_void_p


def P(a):
    return a.ctypes.data_as(_vp)


def _build_oracle():
    so = ROOT / 'oracle' / '_build' / 'libtm_oracle.so'
    if not so.exists():
        subprocess.run(['make', '-s', '-C', str(ROOT / 'oracle')], check=True)
    return so


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        lib = ctypes.CDLL(str(_build_oracle()))
        lib.tmo_cc_to_ed.restype = ctypes.c_float
        lib.tmo_cc_to_ed.argtypes = [ctypes.c_float, ctypes.c_int]
        lib.tmo_ed_to_cc.restype = ctypes.c_float
        lib.tmo_ed_to_cc.argtypes = [ctypes.c_float, ctypes.c_int]
        lib.tmo_l2_dist.restype = ctypes.c_float
        lib.tmo_l2_dist.argtypes = [_vp, _vp, ctypes.c_uint64, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, _vp, _vp]
        lib.tmo_window_stats.argtypes = [_vp, ctypes.c_uint64, ctypes.c_int, _vp, _vp]
        lib.tmo_znormalize.argtypes = [_vp, ctypes.c_int]
        lib.tmo_block_order.argtypes = [_vp, ctypes.c_int, _vp]
        lib.tmo_distance_profile.argtypes = [_vp, ctypes.c_uint64, ctypes.c_int, _vp, _vp]
        lib.tmo_scan_knn.argtypes = [_vp, ctypes.c_uint64, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, _vp, _vp]
        lib.tmo_scan_threshold.restype = ctypes.c_int64
        lib.tmo_scan_threshold.argtypes = [_vp, ctypes.c_uint64, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_float,
                                           ctypes.c_int, _vp, _vp, _vp, ctypes.c_int64]
        lib.tmo_select_knn.argtypes = [_vp, _vp, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, _vp, _vp]
        lib.tmo_window_stats_fast.argtypes = [_vp, ctypes.c_uint64, ctypes.c_int, _vp, _vp]
        _oracle = lib
    return _oracle


def reference():
    """The reference's own SSS build, or None where it was not built."""
    so = ROOT / 'oracle' / '_ref' / 'libtremor_ref.so'
    if not so.exists():
        return None
    lib = ctypes.CDLL(str(so))
    lib.tmref_l2_dist.restype = ctypes.c_float
    lib.tmref_l2_dist.argtypes = [_vp, _vp, ctypes.c_uint64, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_float, _vp, _vp]
    lib.tmref_sss_stats.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, _vp, _vp]
    lib.tmref_znormalize.argtypes = [_vp, ctypes.c_int]
    lib.tmref_block_order.argtypes = [_vp, ctypes.c_int, _vp]
    lib.tmref_sss_knn.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
    lib.tmref_sss_threshold.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, _vp, ctypes.c_int,
                                        ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_char_p]
    lib.tmref_sss_from_stats.restype = _vp
    lib.tmref_sss_from_stats.argtypes = [_vp, ctypes.c_uint64, ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int]
    lib.tmref_sss_search.restype = ctypes.c_double
    lib.tmref_sss_search.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                     ctypes.c_char_p]
    lib.tmref_sss_distances.argtypes = [_vp, _vp, _vp, ctypes.c_uint64, _vp]
    lib.tmref_sss_destroy.argtypes = [_vp]
    return lib


def window_stats_fast(x, m):
    """The reference's per-window (mean, std) floats for a record of any size
    (tmo_window_stats_fast: SkipSequential.cpp:157-190, 32 windows per vector pass)."""
    W = len(x) - m + 1
    mean = np.zeros(W, np.float32)
    std = np.zeros(W, np.float32)
    oracle().tmo_window_stats_fast(P(x), W, m, P(mean), P(std))
    return mean, std


class _QuietStdout:
    """The reference prints per-query timings with printf: keep them off the test output."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.libc = ctypes.CDLL(None)
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


class ReferenceScan:
    """The reference's own SkipSequentialScan (sequential mode, one rank, all host threads)
    over a record in memory, with the statistics of window_stats_fast in place of build()'s
    (tmref_sss_from_stats): for parity checks on records of 2^26-2^28 samples. Answers are
    parsed from the CSV files the reference writes (positions exact, correlations as '%f'
    strings); distances() gives the reference's FP32 distance bits at given windows."""

    def __init__(self, x, m, merge_offset=0, threads=None, stats=None):
        import tempfile
        self.lib = reference()
        if self.lib is None:
            raise RuntimeError('oracle/_ref was not built')
        self.x = np.ascontiguousarray(x, dtype=np.float32)
        self.m = m
        mean, std = stats if stats is not None else window_stats_fast(self.x, m)
        self.tmp = tempfile.TemporaryDirectory()
        with _QuietStdout():
            self.h = self.lib.tmref_sss_from_stats(P(self.x), len(self.x), m, P(mean), P(std), merge_offset,
                                                   threads or os.cpu_count() or 1)
        if not self.h:
            raise RuntimeError('tmref_sss_from_stats failed')

    def _rows(self, path):
        import csv
        with open(path) as f:
            rows = list(csv.reader(f, skipinitialspace=True))
        return [[v.strip() for v in r] for r in rows[1:]]

    def knn(self, templates, k):
        """Per template: (positions uint64[k], correlation strings) as search_knn writes them."""
        q = np.ascontiguousarray(np.atleast_2d(templates), dtype=np.float32)
        out = os.path.join(self.tmp.name, 'knn.csv')
        with _QuietStdout():
            s = self.lib.tmref_sss_search(self.h, P(q), len(q), 1, k, 0.0, out.encode())
        if s < 0:
            raise RuntimeError('reference search_knn failed')
        rows = self._rows(out)
        res = []
        for i in range(len(q)):
            r = [row for row in rows if int(row[0]) == i]
            res.append((np.array([int(row[2]) for row in r], np.uint64), [row[3] for row in r]))
        return res

    def threshold(self, templates, correlation):
        """Per template: (positions, correlation strings) as search_threshold writes them."""
        q = np.ascontiguousarray(np.atleast_2d(templates), dtype=np.float32)
        out = os.path.join(self.tmp.name, 'thr')
        with _QuietStdout():
            s = self.lib.tmref_sss_search(self.h, P(q), len(q), 0, 1, float(correlation), out.encode())
        if s < 0:
            raise RuntimeError('reference search_threshold failed')
        rows = self._rows(out + '_0.csv')
        res = []
        for i in range(len(q)):
            r = [row for row in rows if int(row[0]) == i]
            res.append((np.array([int(row[2]) for row in r], np.uint64), [row[3] for row in r]))
        return res

    def distances(self, template, positions):
        t = np.ascontiguousarray(template, dtype=np.float32)
        pos = np.ascontiguousarray(positions, dtype=np.uint64)
        out = np.zeros(len(pos), np.float32)
        if self.lib.tmref_sss_distances(self.h, P(t), P(pos), len(pos), P(out)) != 0:
            raise RuntimeError('tmref_sss_distances failed')
        return out

    def close(self):
        if getattr(self, 'h', None):
            with _QuietStdout():
                self.lib.tmref_sss_destroy(self.h)
            self.h = None
            self.tmp.cleanup()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def scan_knn(x, queries, m, k, merge):
    q = np.ascontiguousarray(queries, dtype=np.float32)
    I = np.zeros((len(q), k), np.uint64)
    D = np.zeros((len(q), k), np.float32)
    oracle().tmo_scan_knn(P(x), len(x), m, P(q), len(q), k, merge, P(I), P(D))
    return I, D


def scan_threshold(x, queries, m, corr, merge):
    q = np.ascontiguousarray(queries, dtype=np.float32)
    lib = oracle()
    n = lib.tmo_scan_threshold(P(x), len(x), m, P(q), len(q), corr, merge, None, None, None, 0)
    qid = np.zeros(max(n, 1), np.int32)
    pos = np.zeros(max(n, 1), np.uint64)
    dist = np.zeros(max(n, 1), np.float32)
    lib.tmo_scan_threshold(P(x), len(x), m, P(q), len(q), corr, merge, P(qid), P(pos), P(dist), n)
    return qid[:n], pos[:n], dist[:n]


def distance_profile(x, query, m):
    out = np.zeros(len(x) - m + 1, np.float32)
    q = np.ascontiguousarray(query, dtype=np.float32)
    oracle().tmo_distance_profile(P(x), len(x), m, P(q), P(out))
    return out


def ed_to_cc(ed, m):
    return oracle().tmo_ed_to_cc(float(ed), m)


def knn_rows(I, D, m):
    """Rows as the reference's kNN writer prints them (SkipSequential.cpp:461-470)."""
    rows = []
    for qi in range(I.shape[0]):
        for j in range(I.shape[1]):
            rows.append([str(qi), str(j + 1), str(int(I[qi, j])), '%f' % ed_to_cc(D[qi, j], m)])
    return rows


def threshold_rows(qid, pos, dist, m):
    """Rows as the reference's threshold writer prints them (SkipSequential.cpp:313, 367)."""
    rows, counter, last = [], 0, None
    for q, p, d in zip(qid, pos, dist):
        if q != last:
            counter, last = 0, q
        rows.append([str(int(q)), str(counter), str(int(p)), '%f' % ed_to_cc(d, m)])
        counter += 1
    return rows


def golden_cases():
    return sorted(p.stem for p in GOLDEN.glob('*.json'))


def load_golden(name):
    meta = json.loads((GOLDEN / f'{name}.json').read_text())
    arrays = np.load(GOLDEN / f'{name}.npz')
    return meta, arrays['x'], arrays['queries']
