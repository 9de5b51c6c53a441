"""How much could an iSAX lower-bound skip prune on the benchmark workloads? (measurement)

    python oracle/lb_pruning.py [--templates 8]

Uses the reference's own skip-sequential scan (SkipSequentialScan with lower bounds, built
from the reference sources into oracle/_ref by `make -C oracle ref`) on the seeded synthetic
workloads of bench.py: config 1 (2^22 samples, m 1024, kNN k 10, merge 512), config 2 (first
2^24 samples of the 2^26 record, m 2048, correlation >= 0.8) and config 3 (first 2^24 samples
of the 2^28 record, m 4096, kNN k 100). For each template it takes the final bound (the k-th
answer's distance from the reference's own kNN search, or the threshold distance) and counts
the windows whose lower bound does not exceed it: the windows any skip must still compute
exactly. It also reports the share of blocks of 256 consecutive windows (a tensor-core tile's
width) in which no window passes, for one template and for all the sampled templates
together (a 128-template tile could only be skipped where none of its templates passes).
Test infrastructure and a design measurement: nothing in the product imports it."""
from __future__ import annotations

import argparse
import ctypes
import os
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from tests import oracle_bindings as ob  # noqa: E402
from tremor_b200 import synth  # noqa: E402

CONFIGS = [
    ('config 1', dict(n=1 << 22, sample=1 << 22, q=16, m=1024, events=50, k=10, merge=512, corr=None, seed=2026)),
    ('config 2', dict(n=1 << 26, sample=1 << 24, q=256, m=2048, events=500, k=None, merge=0, corr=0.8, seed=2027)),
    ('config 3', dict(n=1 << 28, sample=1 << 24, q=1024, m=4096, events=2000, k=100, merge=0, corr=None, seed=2028)),
]
BLOCK = 256


def main():
    p = argparse.ArgumentParser()
    p.add_argument('--templates', type=int, default=8)
    args = p.parse_args()
    ref = ob.reference()
    if ref is None:
        sys.exit('oracle/_ref not built (make -C oracle ref)')
    ref.tmref_sss_create.restype = ctypes.c_void_p
    ref.tmref_sss_create.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int]
    ref.tmref_sss_lb_pass.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_uint64,
                                      ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
    threads = os.cpu_count() or 1
    print(f'| workload | windows | templates | windows passing the bound (mean, max) | 256-window blocks '
          f'without a passing window: one template (mean) | all sampled templates |')
    print('|---|---|---|---|---|---|')
    for name, c in CONFIGS:
        x, q, _ = synth.workload(c['n'], c['q'], c['m'], c['events'], seed=c['seed'])
        xs = np.ascontiguousarray(x[:c['sample']])
        m = c['m']
        W = len(xs) - m + 1
        nb = (W + BLOCK - 1) // BLOCK
        tpls = q[:args.templates]
        with tempfile.TemporaryDirectory() as tmp:
            wf = os.path.join(tmp, 'w.bin')
            xs.tofile(wf)
            t0 = time.time()
            with ob._QuietStdout():
                h = ref.tmref_sss_create(wf.encode(), len(xs), m, 1, c['merge'], 1, threads, 16)
            build_s = time.time() - t0
            bounds = []
            if c['corr'] is None:  # the k-th answer's distance, from the reference's kNN search
                stats = ob.window_stats_fast(xs, m)
                with ob.ReferenceScan(xs, m, merge_offset=c['merge'], threads=threads, stats=stats) as rs:
                    for (pos, cc) in rs.knn(tpls, c['k']):
                        bounds.append(max(2.0 * m * (1.0 - float(v)) for v in cc) + 2.0 * m * 1e-6)
            else:
                bounds = [2.0 * m * (1.0 - c['corr'])] * len(tpls)
            fracs, empty = [], []
            union = np.zeros(nb, np.uint8)
            for t, b in zip(tpls, bounds):
                any_pass = np.zeros(nb, np.uint8)
                passing = ctypes.c_uint64(0)
                tq = np.ascontiguousarray(t, np.float32)
                assert ref.tmref_sss_lb_pass(h, tq.ctypes.data, b, BLOCK, any_pass.ctypes.data,
                                             ctypes.byref(passing)) == 0
                fracs.append(passing.value / W)
                empty.append(1.0 - any_pass.mean())
                union |= any_pass
            with ob._QuietStdout():
                ref.tmref_sss_destroy(h)
        print(f'| {name}: m {m}, {"kNN k " + str(c["k"]) if c["corr"] is None else "cc >= " + str(c["corr"])}, '
              f'first {len(xs)} samples | {W} | {len(tpls)} | {np.mean(fracs):.4f}, {np.max(fracs):.4f} | '
              f'{np.mean(empty):.4f} | {1.0 - union.mean():.4f} |', flush=True)
        print(f'  (SkipSequentialScan build with lower bounds: {build_s:.1f} s, {threads} threads)', file=sys.stderr)


if __name__ == '__main__':
    main()
