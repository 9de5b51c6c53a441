"""The command-line driver tremor_b200_cli (tremor_b200/cli/tremor_b200_main.cpp): the
reference driver's options and checks (tremor_main.cpp), and on the GPU its CSV files equal
the reference's on the golden fixtures, with the timings CSV beside them."""
import csv
import os
import subprocess
import tempfile
from pathlib import Path

import pytest

from tests import oracle_bindings as ob

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / 'tremor_b200' / 'tremor_b200_cli'


def run(*args):
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True)


def _rows(path):
    with open(path) as f:
        return [[v.strip() for v in r] for r in list(csv.reader(f, skipinitialspace=True))[1:]]


def test_cli_help_and_argument_checks():
    assert run('--help').returncode == 0
    cases = [
        ([], '--dataset is required'),
        (['--dataset', 'd'], '--queries is required'),
        (['--dataset', 'd', '--queries', 'q'], '--window-length must be greater than 0'),
        (['--dataset', 'd', '--queries', 'q', '--window-length', '12'], 'divisible by 8'),
        (['--dataset', 'd', '--queries', 'q', '--window-length', '24'], 'divisible by --paa-segments'),
        (['--dataset', 'd', '--queries', 'q', '--window-length', '64', '--threshold', '1.5'], 'between -1.0 and 1.0'),
        (['--dataset', 'd', '--queries', 'q', '--window-length', '64', '--method', 'fast'], 'Unknown --method'),
        (['--dataset', 'd', '--queries', 'q', '--window-length', '64', '--merge-offset', '-1'], 'non-negative'),
        (['--dataset', 'd', '--queries', 'q', '--window-length', '64', '--bogus'], 'Unknown argument'),
    ]
    for args, message in cases:
        r = run(*args)
        assert r.returncode == 2 and message in r.stderr, (args, r.stderr)


def test_cli_input_checks():
    with tempfile.TemporaryDirectory() as tmp:
        d, q = os.path.join(tmp, 'd.bin'), os.path.join(tmp, 'q.bin')
        open(d, 'wb').write(b'\0' * 4 * 100)
        open(q, 'wb').write(b'\0' * 4 * 70)
        r = run('--dataset', d, '--queries', q, '--window-length', '64')
        assert r.returncode == 1 and 'not divisible by --window-length' in r.stderr
        r = run('--dataset', d, '--queries', q, '--window-length', '128', '--query-count', '1')
        assert r.returncode == 1 and 'fewer samples than --window-length' in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize('name', ob.golden_cases())
def test_cli_writes_reference_csvs(name):
    meta, x, q = ob.load_golden(name)
    with tempfile.TemporaryDirectory() as tmp:
        wf, qf = os.path.join(tmp, 'w.bin'), os.path.join(tmp, 'q.bin')
        x.tofile(wf)
        q.tofile(qf)
        for merge in meta['merges']:
            knn = os.path.join(tmp, f'knn{merge}.csv')
            r = run('--dataset', wf, '--queries', qf, '--window-length', meta['m'], '--paa-segments', 8,
                    '--k', meta['k'], '--merge-offset', merge, '--output', knn, '--method', 'skip-sequential',
                    '--print-knn-results')
            assert r.returncode == 0, r.stderr
            assert _rows(knn) == meta['knn'][str(merge)]
            assert 'KNN search preview' in r.stdout
            timings = _rows(knn + '.timings.csv')
            assert len(timings) == 1 and timings[0][0] == '0' and float(timings[0][2]) > 0
            thr = os.path.join(tmp, f'thr{merge}')
            r = run('--dataset', wf, '--queries', qf, '--window-length', meta['m'], '--paa-segments', 8,
                    '--mode', 'threshold', '--threshold', repr(meta['threshold']), '--merge-offset', merge,
                    '--output', thr, '--no-benchmark-report')
            assert r.returncode == 0, r.stderr
            assert _rows(thr + '_0.csv') == meta['threshold_hits'][str(merge)]
            assert not os.path.exists(thr + '.timings.csv')
