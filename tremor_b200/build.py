"""Builds tremor_b200/libtremor_b200.so (sm_100a) from tremor_b200/csrc.

    python -m tremor_b200.build [--verbose]

nvcc cross-compiles for sm_100a without a GPU; objects go to tremor_b200/_build/.
The host file tm_host.cpp is compiled by g++ with -ffp-contract=off (its arithmetic
must be bit-identical to the reference's; every fused multiply-add is explicit)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / 'csrc'
OUT = HERE / '_build'
LIB = HERE / 'libtremor_b200.so'
CLI = HERE / 'tremor_b200_cli'
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ARCH + ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
                     '-Xcompiler', '-Wall']
CU_SOURCES = ['tm_api.cu', 'tm_stats.cu', 'tm_scan_fp32.cu', 'tm_select.cu', 'tm_scan_umma.cu', 'tm_noalloc.cu',
              'tm_prefix.cu', 'tm_answers.cu', 'tm_groups.cu', 'tm_search.cu', 'tm_serve.cu',
              'tm_probe.cu', 'tm_fp64.cu', 'tm_fftk.cu']
CPP_SOURCES = ['tm_host.cpp']


def _nvcc():
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', shutil.which('nvcc')):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


def _run(cmd, verbose):
    if verbose:
        print(' '.join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'command failed: {" ".join(cmd)}\n{r.stdout}\n{r.stderr}')
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return r.stdout + r.stderr


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    nvcc = _nvcc()
    jobs = []
    for src in CU_SOURCES:
        extra = ['-Xptxas', '-v'] if ptxas_info else []
        jobs.append([nvcc, *NVCC_FLAGS, *extra, '-c', str(CSRC / src), '-o', str(OUT / (src + '.o'))])
    for src in CPP_SOURCES:
        # the image exports CXX pointing at a toolchain without libgomp; use the system g++
        jobs.append(['g++', '-O2', '-std=c++17', '-fPIC', '-ffp-contract=off', '-Wall', '-c', str(CSRC / src),
                     '-o', str(OUT / (src + '.o'))])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        logs = list(ex.map(lambda c: _run(c, verbose), jobs))
    if ptxas_info:
        for log in logs:
            print(log)
    objs = [str(OUT / (s + '.o')) for s in CU_SOURCES + CPP_SOURCES]
    tmp = LIB.with_suffix('.so.tmp')
    _run([nvcc, *ARCH, '-shared', '-o', str(tmp), *objs], verbose)
    os.replace(tmp, LIB)
    # the command-line driver (tremor_main's options and files), next to the library
    cli_tmp = CLI.with_suffix('.tmp')
    _run(['g++', '-O2', '-std=c++17', '-Wall', f'-I{HERE.parent / "include"}', str(HERE / 'cli' / 'tremor_b200_main.cpp'),
          '-o', str(cli_tmp), f'-L{HERE}', '-ltremor_b200', "-Wl,-rpath,$ORIGIN"], verbose)
    os.replace(cli_tmp, CLI)
    return LIB


if __name__ == '__main__':
    build(verbose='--verbose' in sys.argv, ptxas_info='--ptxas' in sys.argv)
    print(LIB)
