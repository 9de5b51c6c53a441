"""The adaptive planner of the reference with its scan and FFT branches on the GPU.

oracle/Makefile builds the reference's whole driver (tremor_main.cpp and the TREMOR engine,
tremor/algos/tremor/*.cpp) from its sources with single-rank MPI and FFTW stand-ins:
`tremor_main_ref` as it is, and `tremor_main_gpu` with the two branch calls of the planner's
worker (Tremor.cpp:2293-2296) routed to tm_gpu_in_position_order
(include/tremor_b200_worker_seam.hpp) by oracle/seam_tremor.py.

* CPU: the reference driver, in leaf order and in adaptive mode, reproduces the golden
  fixtures' CSV files (made by the reference's SkipSequentialScan), which pins the build.
* GPU: `tremor_main_gpu --refinement adaptive --scan-fallback-fraction -1` (every template
  takes the planner's scan branch; the reference's FFT branch is off without FFTW,
  TREMOR_NO_FFT=1) writes the same CSV files, and its output shows the GPU branch answering
  every template.
"""
import csv
import os
import subprocess

import pytest

from tests import oracle_bindings as ob

REF_DRIVER = ob.ROOT / 'oracle' / '_ref' / 'tremor_main_ref'
GPU_DRIVER = ob.ROOT / 'oracle' / '_ref' / 'tremor_main_gpu'


def _rows(path):
    with open(path) as f:
        rows = list(csv.reader(f, skipinitialspace=True))
    return [[v.strip() for v in r] for r in rows[1:]]


def _run(binary, tmp, name, mode, refine, merge):
    """Runs the driver on a golden case; returns (CSV rows, standard output)."""
    meta, x, q = ob.load_golden(name)
    m = meta['m']
    data, queries = tmp / f'{name}.bin', tmp / f'{name}_q.bin'
    if not data.exists():
        x.tofile(data)
        q.astype('float32').tofile(queries)
    out = tmp / f'{name}_{mode}_{refine}_{merge}'
    cmd = [str(binary), '--dataset', str(data), '--queries', str(queries), '--window-length', str(m),
           '--mode', mode, '--k', str(meta['k']), '--threshold', repr(meta['threshold']), '--method', 'tremor',
           '--refinement', refine, '--merge-offset', str(merge),
           '--output', str(out) + ('.csv' if mode == 'knn' else ''), '--search-workers', '4', '--index-threads', '4',
           '--paa-segments', '16' if m % 16 == 0 else '8', '--no-benchmark-report']
    if refine == 'adaptive':
        cmd += ['--scan-fallback-fraction', '-1']
    r = subprocess.run(cmd, capture_output=True, text=True, env=dict(os.environ, TREMOR_NO_FFT='1'), timeout=600)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]
    rows = _rows(str(out) + '.csv') if mode == 'knn' else _rows(str(out) + '_0.csv')
    return rows, r.stdout


def _golden_rows(meta, mode, merge):
    return meta['knn'][str(merge)] if mode == 'knn' else meta['threshold_hits'][str(merge)]


@pytest.mark.skipif(not REF_DRIVER.exists(), reason='reference driver (make -C oracle driver) not built')
@pytest.mark.parametrize('name', ob.golden_cases())
def test_reference_driver_reproduces_golden(name, tmp_path):
    meta, _, q = ob.load_golden(name)
    for merge in meta['merges']:
        for mode in ('knn', 'threshold'):
            for refine in ('leaf', 'adaptive'):
                rows, out = _run(REF_DRIVER, tmp_path, name, mode, refine, merge)
                assert rows == _golden_rows(meta, mode, merge), (name, mode, refine, merge)
                if refine == 'adaptive':
                    assert sum('-> scan' in line for line in out.splitlines()) == len(q)


@pytest.mark.gpu
@pytest.mark.skipif(not GPU_DRIVER.exists(), reason='driver with the GPU seam (make -C oracle driver-gpu) not built')
@pytest.mark.parametrize('name', ob.golden_cases())
def test_gpu_planner_branch_reproduces_golden(name, tmp_path):
    meta, _, q = ob.load_golden(name)
    for merge in meta['merges']:
        for mode in ('knn', 'threshold'):
            rows, out = _run(GPU_DRIVER, tmp_path, name, mode, 'adaptive', merge)
            assert rows == _golden_rows(meta, mode, merge), (name, mode, merge)
            assert sum('GPU branch' in line for line in out.splitlines()) == len(q), out[-2000:]
