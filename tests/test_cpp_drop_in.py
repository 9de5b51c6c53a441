"""The C++ drop-in class GpuSkipSequentialScan (include/tremor_b200_sss.hpp), used the way
the reference's driver uses SkipSequentialScan, writes the reference's CSV files with the
reference's answers (golden fixtures). The build runs on CPU; the run needs the GPU."""
import csv
import os
import subprocess
import tempfile
from pathlib import Path

import pytest

from tests import oracle_bindings as ob

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / 'tests' / 'cpp' / 'sss_drop_in.cpp'


def build_driver(out_dir):
    exe = os.path.join(out_dir, 'sss_drop_in')
    subprocess.run(['g++', '-O2', '-std=c++17', f'-I{ROOT / "include"}', str(SRC), '-o', exe,
                    f'-L{ROOT / "tremor_b200"}', '-ltremor_b200', f'-Wl,-rpath,{ROOT / "tremor_b200"}'],
                   check=True)
    return exe


def test_drop_in_class_compiles_and_links():
    with tempfile.TemporaryDirectory() as tmp:
        assert os.path.exists(build_driver(tmp))


def _rows(path):
    with open(path) as f:
        return [[v.strip() for v in r] for r in list(csv.reader(f, skipinitialspace=True))[1:]]


@pytest.mark.gpu
@pytest.mark.parametrize('name', ob.golden_cases())
def test_drop_in_class_writes_reference_csvs(name):
    meta, x, q = ob.load_golden(name)
    with tempfile.TemporaryDirectory() as tmp:
        exe = build_driver(tmp)
        wf, qf = os.path.join(tmp, 'w.bin'), os.path.join(tmp, 'q.bin')
        x.tofile(wf)
        q.tofile(qf)
        for merge in meta['merges']:
            out = os.path.join(tmp, f'o{merge}')
            subprocess.run([exe, wf, str(len(x)), str(meta['m']), qf, str(len(q)), str(meta['k']), str(merge),
                            repr(meta['threshold']), out], check=True)
            assert _rows(out + '.knn.csv') == meta['knn'][str(merge)]
            assert _rows(out + '.thr_0.csv') == meta['threshold_hits'][str(merge)]
