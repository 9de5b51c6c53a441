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
    return lib


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
