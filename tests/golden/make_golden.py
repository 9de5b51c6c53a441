"""Generates the golden fixtures of tests/golden/ from the reference's OWN scan code.

Run where the reference sources are mounted (REF; default: the `reference` checkout
beside this repository):  python tests/golden/make_golden.py

It builds oracle/_ref/libtremor_ref.so (the reference's SkipSequentialScan with a
single-rank MPI stand-in, see oracle/Makefile), runs it on seeded inputs and
writes, per case, the inputs (<case>.npz) and the reference's answers exactly as
its CSV writers print them (<case>.json). The tests compare the oracle and the
GPU library with these answers; they never need the reference at run time.

Cases:
  validate     the seeded case of experiments/validate_search.py:50-76 (seed 734,
               n=8192, m=64, k=5, threshold 0.4, merge 0 and m/4; a constant
               stretch, a 1e6-loud stretch followed by a 1e-3-quiet one; windows at
               the first/last positions and one random template)
  tail_missing m=72 (a 32-sample block order plus an 8-sample tail), missing samples
               (-100000) scattered and in a run, windows that start on one
  sparse       so few windows that the kNN bound never fills (2k-1 > separated
               windows), with a constant stretch: padded and FLT_MAX answers
  chirp        the seeded AR(2)+chirp generator, k=10 / merge m/2, threshold 0.8
"""
from __future__ import annotations

import csv
import ctypes
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from tremor_b200 import synth  # noqa: E402


def cases():
    out = {}
    # experiments/validate_search.py:50-57, 75-77
    rng = np.random.default_rng(734)
    n, m = 8192, 64
    x = rng.normal(size=n).astype('float32')
    x[2000:2128] = 0
    x[5000:6000] *= 1e6
    x[6000:6600] *= 1e-3
    positions = [0, 4090, min(6200, n - m - 1), n - m]
    queries = np.stack([x[p:p + m] for p in positions] + [rng.normal(size=m)]).astype('float32')
    out['validate'] = dict(x=x, queries=queries, m=m, k=5, merges=[0, m // 4], threshold=0.4, paa=8)

    rng = np.random.default_rng(2029)
    n, m = 6000, 72
    x = (rng.normal(size=n) * 3 + 1).astype('float32')
    x[rng.integers(0, n, 40)] = synth.MISSING_VALUE
    x[3000:3050] = synth.MISSING_VALUE
    x[1500:1600] = 7.0
    pos = [10, 2990, 4000, n - m]
    queries = np.stack([x[p:p + m] for p in pos] + [rng.normal(size=m)]).astype('float32')
    queries[queries == synth.MISSING_VALUE] = 0.5
    out['tail_missing'] = dict(x=x, queries=queries, m=m, k=7, merges=[0, m // 2], threshold=0.3, paa=8)

    rng = np.random.default_rng(2031)
    n, m = 400, 64
    x = rng.normal(size=n).astype('float32')
    x[100:200] = 3.0
    queries = np.stack([x[20:20 + m], rng.normal(size=m)]).astype('float32')
    out['sparse'] = dict(x=x, queries=queries, m=m, k=10, merges=[0, 64], threshold=-0.5, paa=8)

    x, queries, _ = synth.workload(1 << 15, 4, 256, 12, seed=2027)
    out['chirp'] = dict(x=x, queries=queries, m=256, k=10, merges=[0, 128], threshold=0.8, paa=16)
    return out


def read_csv(path):
    with open(path) as f:
        rows = list(csv.reader(f, skipinitialspace=True))
    return [[v.strip() for v in r] for r in rows[1:]]


def main():
    ref = os.environ.get('REF', str(ROOT.parent / 'reference'))
    subprocess.run(['make', '-C', str(ROOT / 'oracle'), 'ref', f'REF={ref}'], check=True)
    lib = ctypes.CDLL(str(ROOT / 'oracle' / '_ref' / 'libtremor_ref.so'))
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    for name, c in cases().items():
        x, q, m = c['x'], c['queries'], c['m']
        np.savez_compressed(HERE / f'{name}.npz', x=x, queries=q)
        result = dict(case=name, n=len(x), m=m, k=c['k'], threshold=c['threshold'], merges=c['merges'],
                      query_count=len(q), knn={}, threshold_hits={})
        with tempfile.TemporaryDirectory() as tmp:
            wf = os.path.join(tmp, 'waveform.bin')
            x.tofile(wf)
            for merge in c['merges']:
                out = os.path.join(tmp, f'knn{merge}.csv')
                rc = lib.tmref_sss_knn(wf.encode(), ctypes.c_uint64(len(x)), m, P(q), len(q), c['k'], merge, 0, 4,
                                       c['paa'], out.encode())
                assert rc == 0, name
                result['knn'][str(merge)] = read_csv(out)
                prefix = os.path.join(tmp, f'thr{merge}')
                rc = lib.tmref_sss_threshold(wf.encode(), ctypes.c_uint64(len(x)), m, P(q), len(q),
                                             ctypes.c_float(c['threshold']), merge, 0, 4, c['paa'], prefix.encode())
                assert rc == 0, name
                result['threshold_hits'][str(merge)] = read_csv(prefix + '_0.csv')
        (HERE / f'{name}.json').write_text(json.dumps(result, indent=1) + '\n')
        print(name, {k: len(v) for k, v in result['threshold_hits'].items()})


if __name__ == '__main__':
    main()
