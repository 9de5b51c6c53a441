"""Benchmark of the exact template-matching scan on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload precision|plain_knn|threshold|...] [--kernel auto|fp32|bf16]

Workload (default "precision"): a seeded synthetic waveform of 2^28 float32 samples
(AR(2) noise x slow envelope, 2000 injected chirp events), 1024 chirp templates of
4096 samples, kNN k=100 with merge offset 0. One step = one batch of 128 templates
against every window of the waveform (2^28 - 4095 windows); the metric is
template-subsequence pairs per second (G pairs/s), whole job over all GPUs.

`value`: templates already resident in HBM (a prepared batch), each step the full
device pipeline plus the exact answers copied back. `e2e`: the same steps through
the public call with host templates (host z-normalisation, host->device copy,
device pipeline, device->host answers). The waveform (1 GiB) is larger than L2, so
no flush is needed between steps. With N GPUs every rank runs its own replica (the
path needs no exchange); time is the max over ranks.

After the timed legs, untimed: every answer of one step is recomputed in FP64
(`fp64_error`: the error against FP64 stated per result, summarised), and the plain FP32
kernel runs the same batches (`plain_fp32`, at most 3 steps); `vs_baseline` is value over
that FP32 rate, the metric's own comparison. Then a short serving leg (`serving`: config 5's
2^29-sample record, 150 requests at 200 req/s, p50/p99 latency and the achieved rate).

--impl reference: the reference's own CPU scan (SkipSequentialScan, sequential mode,
built from the reference sources into oracle/_ref) on a bounded sample of the same
workload (the first 2^24 samples, a few templates per step), all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = 'G template-subseq pairs/s vs plain FP32 kernel, exact answers; p50/p99 latency'
UNIT = 'G pairs/s'

WORKLOADS = {
    # precision = config 3, plain_knn = config 1, threshold = config 2
    # config 3 names the contraction: split-BF16 tensor cores (the default kernel here)
    'precision': dict(n=1 << 28, q=1024, m=4096, events=2000, mode='knn', k=100, merge=0, corr=0.0,
                      per_step=128, seed=2028, kernel='bf16', serving_leg=True),
    'plain_knn': dict(n=1 << 22, q=16, m=1024, events=50, mode='knn', k=10, merge=512, corr=0.0,
                      per_step=16, seed=2026),
    # the precision workload's kernel on 2^25 samples (> L2) and 64 templates: ncu captures
    'precision_small': dict(n=1 << 25, q=64, m=4096, events=250, mode='knn', k=100, merge=0, corr=0.0,
                            per_step=64, seed=2028),
    'threshold': dict(n=1 << 26, q=256, m=2048, events=500, mode='threshold', k=1, merge=0, corr=0.8,
                      per_step=256, seed=2027),
    # config 4: lengths log-uniform in [256, 8192] (multiples of 16), random centre
    # frequencies, 50/50 kNN (k in {1, 10, 100}, merge m/2) and threshold (0.6-0.9); the
    # whole batch is one step (one mixed-length launch)
    'batching': dict(n=1 << 27, q=4096, m=(256, 8192), events=2000, mode='mixed', k=0, merge=0, corr=0.0,
                     per_step=4096, seed=2029),
    'batching_small': dict(n=1 << 25, q=512, m=(256, 8192), events=250, mode='mixed', k=0, merge=0, corr=0.0,
                           per_step=512, seed=2029),
    # few long templates (the FFT branch's case): 2^28 samples, 8 chirps of 16384, kNN k=10
    'long_templates': dict(n=1 << 28, q=8, m=16384, events=200, mode='knn', k=10, merge=8192, corr=0.0,
                           per_step=8, seed=2031),
    # the FFT branch's kernel on 2^25 samples (inputs > L2): ncu captures
    'fft_small': dict(n=1 << 25, q=8, m=8192, events=50, mode='knn', k=10, merge=4096, corr=0.0,
                      per_step=8, seed=2032),
    # the fused in-tree FFT branch (templates up to 8192): 2^28 samples, 8 chirps of 8192
    'fft_templates': dict(n=1 << 28, q=8, m=8192, events=200, mode='knn', k=10, merge=4096, corr=0.0,
                          per_step=8, seed=2032),
    # config 5: 2^29 samples resident with their prefix sums; a Poisson stream of requests
    # (lengths log-uniform in [128, 16384], 50/50 kNN / threshold as in config 4) served
    # with continuous batching; one step = one request
    'serving': dict(n=1 << 29, q=1024, m=(128, 16384), events=4000, mode='mixed', k=0, merge=0, corr=0.0,
                    per_step=1, seed=2030, serve=True, requests=400, rate=200.0),
    'serving_small': dict(n=1 << 26, q=256, m=(128, 16384), events=500, mode='mixed', k=0, merge=0, corr=0.0,
                          per_step=1, seed=2030, serve=True, requests=200, rate=200.0),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_workload(w):
    from tremor_b200 import synth
    t0 = time.time()
    if w['mode'] == 'mixed':
        x, q, _ = synth.mixed_workload(w['n'], w['q'], w['m'][0], w['m'][1], w['events'], seed=w['seed'])
    else:
        x, q, _ = synth.workload(w['n'], w['q'], w['m'], w['events'], seed=w['seed'])
    log(f'[bench] workload generated in {time.time() - t0:.1f} s')
    return x, q


def requests_for(w, q):
    import tremor_b200 as tb
    if w['mode'] == 'mixed':
        rng = np.random.default_rng(w['seed'] + 1)
        reqs = []
        for i, t in enumerate(q):
            if i % 2 == 0:
                reqs.append(tb.Request(t, tb.MODE_KNN, k=int(rng.choice([1, 10, 100])), merge_offset=len(t) // 2))
            else:
                reqs.append(tb.Request(t, tb.MODE_THRESHOLD, correlation=float(rng.uniform(0.6, 0.9))))
        return reqs
    if w['mode'] == 'knn':
        return [tb.Request(t, tb.MODE_KNN, k=w['k'], merge_offset=w['merge']) for t in q]
    return [tb.Request(t, tb.MODE_THRESHOLD, correlation=w['corr'], merge_offset=w['merge']) for t in q]


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device):
        self.device, self.proc, self.lines = device, None, []
        self.first = threading.Event()

    WARM_SAMPLES = 3

    def start(self):
        """Starts sampling and returns once the first WARM_SAMPLES samples are in (at most
        10 s): NVML's start-up in nvidia-smi can hold the driver for about a second, which
        must not fall inside the timed region."""
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.device), f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            self.first.wait(timeout=10.0)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            if len(self.lines) >= self.WARM_SAMPLES:
                self.first.set()
        self.first.set()

    def stop(self):
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, power, reasons = [], None, [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.lines:
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith('active'):
                    reasons.add(name)
        loaded = [s for s, p in zip(sm, power) if p > 300] or sm
        return {'sm_mhz': statistics.median(loaded) if loaded else None, 'sm_max_mhz': smax,
                'reasons': sorted(reasons), 'samples': len(sm), 'power_w_max': max(power) if power else None}


def peaks():
    path = ROOT / 'MEASURED_PEAKS.json'
    if path.exists():
        d = json.loads(path.read_text())
        return d.get('bf16_tflops', 1590.0), d.get('hbm_gbs', 6650.0), 'measured'
    return 1590.0, 6650.0, 'fallback'


def peaks_sustained():
    """The measured sustained BF16 figure (a seconds-long GEMM loop under the power cap),
    or None."""
    path = ROOT / 'MEASURED_PEAKS.json'
    if path.exists():
        return json.loads(path.read_text()).get('bf16_tflops_sustained')
    return None


def traffic_for(kernel, workload):
    """Per-launch DRAM bytes of the kernel from the committed ncu summary, or None."""
    path = ROOT / 'profiles' / 'traffic.txt'
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
            return float(parts[2])
    return None


class _StdoutToStderr:
    """While active, the process's C-level standard output goes to standard error: the
    reference library prints per-query timings with printf, and standard output must carry
    the one JSON line only."""

    def __enter__(self):
        import ctypes
        sys.stdout.flush()
        self.libc = ctypes.CDLL(None)
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)


class RefScan:
    """The reference's own SkipSequentialScan (sequential mode, no lower bounds) built once on
    the first 2^24 samples of the waveform (its build is the reference's index step, not
    timed); search() times SkipSequentialScan::search_knn / search_threshold alone."""

    def __init__(self, w, x, m=None, threads=None, lower_bounds=False):
        import ctypes
        from tests import oracle_bindings as ob
        self.w, self.ct, self.h = w, ctypes, None
        self.ref = ob.reference()
        if self.ref is None:
            self.error = 'oracle/_ref not built'
            return
        ref = self.ref
        ref.tmref_sss_create.restype = ctypes.c_void_p
        ref.tmref_sss_create.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int]
        ref.tmref_sss_search.restype = ctypes.c_double
        ref.tmref_sss_search.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_float, ctypes.c_char_p]
        ref.tmref_sss_destroy.argtypes = [ctypes.c_void_p]
        self.threads = threads or os.cpu_count() or 1
        n_s = min(len(x), 1 << 24)
        self.m = m = m if m is not None else w['m']
        self.windows = n_s - m + 1
        self.tmp = tempfile.TemporaryDirectory()
        wf = os.path.join(self.tmp.name, 'w.bin')
        x[:n_s].tofile(wf)
        t0 = time.time()
        with _StdoutToStderr():
            self.h = ref.tmref_sss_create(wf.encode(), n_s, m, w['k'], w['merge'], 1 if lower_bounds else 0,
                                          self.threads, 16 if m % 16 == 0 else 8)
        log(f'[bench] reference scan built in {time.time() - t0:.1f} s ({self.threads} threads)')
        self.error = None if self.h else 'reference build failed'

    def search(self, template) -> float:
        qi = np.ascontiguousarray(np.asarray(template, np.float32)[None, :])
        out = os.path.join(self.tmp.name, 'out.csv')
        knn = self.w['mode'] != 'threshold'
        with _StdoutToStderr():
            s = self.ref.tmref_sss_search(self.h, qi.ctypes.data_as(self.ct.c_void_p), 1, 1 if knn else 0,
                                          max(self.w['k'], 10), self.w['corr'], out.encode())
        if s < 0:
            raise RuntimeError('reference search failed')
        return s

    def close(self):
        if self.h:
            with _StdoutToStderr():
                self.ref.tmref_sss_destroy(self.h)
            self.h = None


def sample_templates(w, q):
    """Templates of the CPU sample: all of them for single-length workloads; for the
    mixed-length workload three templates spread over the lengths (one build each)."""
    if w['mode'] != 'mixed':
        return list(q)
    order = sorted(range(len(q)), key=lambda i: len(q[i]))
    return [q[order[len(order) * f // 4]] for f in (1, 2, 3)]


def cpu_reference(w, x, q, budget_s=15.0, max_templates=32):
    """(pairs/s, info) of the reference's CPU scan over a bounded sample: as many templates as
    fit in about `budget_s` seconds of search, at least one."""
    tpls = sample_templates(w, q)
    done, secs, pairs, threads = 0, 0.0, 0, 1
    scans = {}
    try:
        while done < min(max_templates, len(tpls)) and (secs < budget_s or done == 0):
            t = tpls[done]
            if len(t) not in scans:
                scans[len(t)] = RefScan(w, x, m=len(t))
                if scans[len(t)].error:
                    return None, {'error': scans[len(t)].error}
            scan = scans[len(t)]
            secs += scan.search(t)
            pairs += scan.windows
            threads = scan.threads
            done += 1
    finally:
        for scan in scans.values():
            scan.close()
    info = {'cores': threads, 'kind': 'reference',
            'sample': f'{done} templates x ~{pairs // max(done, 1)} windows (first 2^24 samples of the waveform), '
                      f'SkipSequentialScan sequential mode, {secs:.1f} s of search'}
    # the skip-sequential mode (iSAX lower bounds prune windows) on the same sample
    try:
        secs_lb, pairs_lb, done_lb = 0.0, 0, 0
        scan = None
        for t in tpls[:done]:
            if scan is None or scan.m != len(t):
                if scan is not None:
                    scan.close()
                scan = RefScan(w, x, m=len(t), lower_bounds=True)
                if scan.error:
                    raise RuntimeError(scan.error)
            secs_lb += scan.search(t)
            pairs_lb += scan.windows
            done_lb += 1
            if secs_lb > budget_s:
                break
        if scan is not None:
            scan.close()
        info['skip_sequential'] = {'value': pairs_lb / secs_lb / 1e9, 'unit': UNIT, 'cores': threads,
                                   'sample': f'{done_lb} templates, same windows, {secs_lb:.1f} s of search'}
    except Exception as exc:  # informative leg
        info['skip_sequential'] = {'error': str(exc)[:200]}
    return pairs / secs / 1e9, info


def cpu_mass(w, x, q, budget_s=8.0, max_templates=8):
    """(pairs/s, info) of the reference's MASS V3 (dmass/DMASS_V3.c, restated in
    oracle/mass_v3.py with scipy's pocketfft for FFTW) on the first 2^24 samples, all host
    threads; its set-up (piece spectra, statistics) is not timed."""
    sys.path.insert(0, str(ROOT / 'oracle'))
    from mass_v3 import MassV3
    n_s = min(len(x), 1 << 24)
    tpls = sample_templates(w, q)
    done, secs, pairs, workers = 0, 0.0, 0, 1
    masses = {}
    while done < min(max_templates, len(tpls)) and (secs < budget_s or done == 0):
        t = tpls[done]
        if len(t) not in masses:
            t0 = time.time()
            masses[len(t)] = MassV3(x[:n_s], len(t))
            log(f'[bench] MASS V3 set up in {time.time() - t0:.1f} s (m={len(t)})')
        mass = masses[len(t)]
        t0 = time.perf_counter()
        mass.distances(t)
        secs += time.perf_counter() - t0
        pairs += mass.W
        workers = mass.workers
        done += 1
    return pairs / secs / 1e9, {'cores': workers, 'kind': 'port', 'fft': 'scipy.fft pocketfft, double precision',
                                'sample': f'{done} templates x ~{pairs // max(done, 1)} windows (first 2^24 samples), '
                                          f'{secs:.1f} s of queries'}


def dist_setup(gpus):
    if gpus <= 1 or 'RANK' not in os.environ:
        return 0, 1, int(os.environ.get('LOCAL_RANK', 0)), None
    import datetime
    import torch.distributed as dist
    dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
    return dist.get_rank(), dist.get_world_size(), int(os.environ.get('LOCAL_RANK', 0)), dist


def run_reference(args, w):
    rank, world, local, dist = dist_setup(args.gpus)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    x, q = make_workload(w)  # the sample is the first 2^24 samples of the full waveform
    tpls = sample_templates(w, q)
    scans = {}
    for t in tpls:
        if len(t) not in scans:
            scans[len(t)] = RefScan(w, x, m=len(t))
            if scans[len(t)].error:
                print(json.dumps({'impl': 'reference', 'unavailable': scans[len(t)].error}), flush=True)
                return
    per_step = max(1, int(os.environ.get('TM_REF_TEMPLATES_PER_STEP', 2)))
    for s in range(args.warmup):
        t = tpls[s % len(tpls)]
        scans[len(t)].search(t)
    secs, pairs = 0.0, 0
    for s in range(args.steps):
        for i in range(per_step):
            t = tpls[(s * per_step + i) % len(tpls)]
            secs += scans[len(t)].search(t)
            pairs += scans[len(t)].windows
    for scan in scans.values():
        scan.close()
    scan = next(iter(scans.values()))
    value = pairs / secs / 1e9
    info = {'cores': scan.threads, 'kind': 'reference',
            'sample': f'{per_step} templates x {scan.windows} windows per step (first 2^24 samples), '
                      'SkipSequentialScan sequential mode'}
    line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': args.gpus, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1000.0 * secs / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'impl': 'reference',
            'config': {'workload': args.workload, **{k: w[k] for k in ('n', 'q', 'm', 'k', 'merge', 'corr')},
                       'sample': 'first 2^24 samples'},
            'cpu_baseline': {'value': value, 'unit': UNIT, **info},
            'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_serving(args, w):
    """Config 5: a Poisson stream of requests against a served context. Throughput is total
    pairs over the span from the first submission to the last completion (the server's
    steady clock); latency is completion minus submission per request. Warm-up requests
    are served and discarded first."""
    import threading as th
    import torch
    import tremor_b200 as tb
    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    x, q = make_workload(w)
    reqs = requests_for(w, q)
    rate = args.rate or w['rate']
    count = args.requests or w['requests']
    rng = np.random.default_rng(w['seed'] + 2 + rank)
    pick = rng.integers(0, len(reqs), size=count)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=count))
    ctx = tb.Context(x, device=local)
    t0 = time.time()
    server = ctx.serve(workers=args.workers, max_batch=args.max_batch, batch_ms=args.batch_ms)
    log(f'[bench] server started (prefix sums) in {time.time() - t0:.2f} s')
    for s in range(args.warmup):  # untimed: a few batches of 8 requests
        for i in range(8):
            server.submit(reqs[(s * 8 + i) % len(reqs)])
        got = 0
        while got < 8:
            got += len(server.poll(64, 1000))
    launches0 = server.status()[3]
    sampler = ClockSampler(local)
    sampler.start()
    if dist:
        dist.barrier()
    tickets = {}

    def submitter():
        start = time.perf_counter()
        for i in range(count):
            delay = arrivals[i] - (time.perf_counter() - start)
            if delay > 0:
                time.sleep(delay)
            tickets[server.submit(reqs[pick[i]])] = i

    sub = th.Thread(target=submitter)
    sub.start()
    done = {}
    while len(done) < count:
        for c in server.poll(256, 500):
            done[c.ticket] = c
    sub.join()
    clocks = sampler.stop()
    launches = server.status()[3] - launches0
    server.stop()
    comps = list(done.values())
    bad = [c for c in comps if c.status != 0]
    if bad:
        raise RuntimeError(f'{len(bad)} served requests failed (status {bad[0].status})')
    span_ms = max(c.done_ms for c in comps) - min(c.submit_ms for c in comps)
    lens = [len(reqs[pick[tickets[c.ticket]]].template) for c in comps]
    pairs = sum(w['n'] - m + 1 for m in lens)
    flops = sum(2.0 * m * (w['n'] - m + 1) for m in lens)
    lat = np.array([c.done_ms - c.submit_ms for c in comps])
    queue = np.array([c.start_ms - c.submit_ms for c in comps])
    service = np.array([c.done_ms - c.start_ms for c in comps])
    answers = sum(len(c.answers[0]) for c in comps)
    from tremor_b200.replicas import combine
    dev = f'cuda:{local}'
    pairs_all, span_ms = combine(pairs, span_ms, dist, dev)  # all work, the slowest rank's span
    flops_all, _ = combine(flops, span_ms, dist, dev)
    value = pairs_all / (span_ms / 1e3) / 1e9
    if rank == 0:
        bf16_peak, _, peak_kind = peaks()
        achieved = flops_all / world / (span_ms / 1e3) / 1e12
        roof = {'bound': 'tensor', 'achieved': achieved, 'peak': bf16_peak / 3.0, 'unit': 'TFLOP/s',
                'frac': achieved / (bf16_peak / 3.0), 'traffic': None, 'kernel': 'k_scan_umma',
                'peak_note': f'{peak_kind} bf16 dense / 3; achieved = algorithmic flops over the whole '
                             'serving span (a lower bound on the kernel rate: queue gaps included)'}
        cpu_v, cpu_info = (None, {'error': 'skipped'}) if args.no_cpu else cpu_reference(w, x, q)
        pct = lambda a, p: float(np.percentile(a, p))
        line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': count,
                'warmup': args.warmup, 'ms_per_step': span_ms / count, 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'bf16x3+f32', 'data': 'synthetic',
                'config': {'workload': args.workload, 'n': w['n'], 'templates': w['q'], 'm': w['m'],
                           'requests': count, 'arrival': f'poisson {rate} req/s', 'seed': w['seed'],
                           'workers': args.workers, 'max_batch': args.max_batch, 'batch_ms': args.batch_ms,
                           'l2': 'inputs larger than L2 (waveform 4n bytes)', 'parallelism': f'replicas x{world}',
                           'timing': 'server steady clock, first submission to last completion'},
                'latency_ms': {'p50': pct(lat, 50), 'p99': pct(lat, 99), 'mean': float(lat.mean()),
                               'queue_p50': pct(queue, 50), 'queue_p99': pct(queue, 99),
                               'service_p50': pct(service, 50), 'service_p99': pct(service, 99)},
                'offered_rate_rps': rate, 'achieved_rate_rps': count / (span_ms / 1e3),
                'batch_size': {'mean': float(np.mean([c.batch_size for c in comps])),
                               'max': int(max(c.batch_size for c in comps))},
                'roofline': roof,
                'cpu_baseline': {'value': cpu_v, 'unit': UNIT, **cpu_info},
                'e2e': {'value': value, 'unit': UNIT,
                        'h2d_bytes_per_step': int(4 * sum(lens) / count),
                        'd2h_bytes_per_step': int(8 * answers / count)},
                'gpu_launches': launches, 'clocks': clocks}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def serving_leg(local, rate=200.0, count=150, batch_ms=0.0):
    """Config 5 in brief, for the default bench line: the serving workload's record (2^29
    samples, resident with its prefix sums) and a Poisson stream of `count` requests at `rate`
    req/s (lengths log-uniform 128-16384, 50/50 kNN / threshold), after 8 untimed warm-up
    requests. Latency is completion minus submission (the server's steady clock); throughput
    is all pairs over the span from the first submission to the last completion."""
    import threading as th
    import tremor_b200 as tb
    w = WORKLOADS['serving']
    x, q = make_workload(w)
    reqs = requests_for(w, q)
    rng = np.random.default_rng(w['seed'] + 2)
    pick = rng.integers(0, len(reqs), size=count)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=count))
    with tb.Context(x, device=local) as ctx:
        server = ctx.serve(batch_ms=batch_ms)
        for i in range(8):
            server.submit(reqs[i])
        got = 0
        while got < 8:
            got += len(server.poll(64, 1000))
        tickets = {}

        def submitter():
            start = time.perf_counter()
            for i in range(count):
                delay = arrivals[i] - (time.perf_counter() - start)
                if delay > 0:
                    time.sleep(delay)
                tickets[server.submit(reqs[pick[i]])] = i

        sub = th.Thread(target=submitter)
        sub.start()
        done = {}
        while len(done) < count:
            for c in server.poll(256, 500):
                done[c.ticket] = c
        sub.join()
        server.stop()
    comps = list(done.values())
    if any(c.status != 0 for c in comps):
        raise RuntimeError('a served request failed')
    span_ms = max(c.done_ms for c in comps) - min(c.submit_ms for c in comps)
    lens = [len(reqs[pick[tickets[c.ticket]]].template) for c in comps]
    lat = np.array([c.done_ms - c.submit_ms for c in comps])
    return {'workload': 'serving (config 5): 2^29 samples, lengths 128-16384, 50/50 kNN / threshold',
            'requests': count, 'offered_rate_rps': rate, 'achieved_rate_rps': count / (span_ms / 1e3),
            'value': sum(w['n'] - m + 1 for m in lens) / (span_ms / 1e3) / 1e9, 'unit': UNIT,
            'latency_ms': {'p50': float(np.percentile(lat, 50)), 'p99': float(np.percentile(lat, 99)),
                           'mean': float(lat.mean())},
            'batch_size_mean': float(np.mean([c.batch_size for c in comps])), 'batch_ms': batch_ms}


def run_ours(args, w):
    import torch
    import tremor_b200 as tb
    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    x, q = make_workload(w)
    if args.kernel is None:
        args.kernel = w.get('kernel', 'auto')
    kernel = {'auto': tb.KERNEL_AUTO, 'fp32': tb.KERNEL_FP32, 'bf16': tb.KERNEL_SPLIT_BF16}[args.kernel]
    ctx = tb.Context(x, device=local)
    ctx.set_kernel(kernel)
    ctx.set_tiles({'auto': tb.TILES_AUTO, 'rows': tb.TILES_ROWS, 'cols128': tb.TILES_COLS_128,
                   'cols64': tb.TILES_COLS_64, 'cols32': tb.TILES_COLS_32}[args.tiles])
    t0 = time.time()
    if w['mode'] != 'mixed':
        ctx.prepare_length(w['m'])
    log(f'[bench] window statistics in {time.time() - t0:.2f} s')
    reqs = requests_for(w, q)
    per = w['per_step']
    nbatch = (len(reqs) + per - 1) // per
    batches = [ctx.batch(reqs[i * per:(i + 1) * per]) for i in range(nbatch)]
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local)
    pair_count = [sum(w['n'] - len(r.template) + 1 for r in reqs[i * per:(i + 1) * per]) for i in range(nbatch)]

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    # the sampler starts first: its start-up must not leave the GPU idle (clocks ramping
    # down) between the warm-up and the timed steps
    sampler = ClockSampler(local)
    sampler.start()
    for s in range(args.warmup):
        batches[s % nbatch].run()
    ctx.profile_enable(True)
    ctx.profile_read()
    ctx.profile_phases()
    ctx.d2h_bytes()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    pairs = 0
    step_ev, step_host = [ev0], []
    for s in range(args.steps):
        b = batches[(args.warmup + s) % nbatch]
        h0 = time.perf_counter()
        b.run()
        step_host.append(1000 * (time.perf_counter() - h0))
        pairs += pair_count[(args.warmup + s) % nbatch]
        if s + 1 < args.steps:
            step_ev.append(torch.cuda.Event(enable_timing=True))
            step_ev[-1].record(stream)
    ev1.record(stream)
    step_ev.append(ev1)
    barrier()
    clocks = sampler.stop()
    log('[bench] steps (device ms / host run ms): ' +
        ', '.join(f'{a.elapsed_time(b):.1f}/{h:.1f}' for a, b, h in zip(step_ev, step_ev[1:], step_host)))
    ms = ev0.elapsed_time(ev1)
    kname, launches, kms, kflops, all_launches = ctx.profile_read()
    phase_ms = {k: v / args.steps for k, v in ctx.profile_phases().items()}
    ctx.profile_enable(False)
    log('[bench] phases per step (ms): ' + ', '.join(f'{k} {v:.1f}' for k, v in phase_ms.items()))
    d2h_value = ctx.d2h_bytes()

    # e2e: host templates through the public call, copies inside the timed region
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h2d = 0
    e0.record(stream)
    phases = [0.0, 0.0, 0.0]
    for s in range(args.steps):
        chunk = reqs[((args.warmup + s) % nbatch) * per:((args.warmup + s) % nbatch + 1) * per]
        t0 = time.perf_counter()
        b = ctx.batch(chunk)
        t1 = time.perf_counter()
        h2d += b.h2d_bytes()
        b.run()
        t2 = time.perf_counter()
        b.close()
        t3 = time.perf_counter()
        phases = [phases[0] + t1 - t0, phases[1] + t2 - t1, phases[2] + t3 - t2]
    e1.record(stream)
    barrier()
    e_ms = e0.elapsed_time(e1)
    d2h = ctx.d2h_bytes()
    log('[bench] e2e host phases per step (create, run, close) ms: ' +
        ', '.join(f'{1000 * p / args.steps:.1f}' for p in phases))

    # the error of every answer of one step against FP64 (tm_result_fp64), untimed
    ans = batches[0].run(fp64=True)
    rel = np.concatenate([tb.Context.relative_error(d, f) for _, d, f in ans])
    d64 = np.concatenate([f for _, _, f in ans])
    fin = rel[np.isfinite(rel)]
    fp64_error = {'answers': int(len(rel)), 'finite': int(len(fin)),
                  'max_rel': float(fin.max()) if len(fin) else None,
                  'median_rel': float(np.median(fin)) if len(fin) else None,
                  'min_fp64_distance': float(d64[np.isfinite(d64)].min()) if np.isfinite(d64).any() else None,
                  'within_1e-4': int((fin <= 1e-4).sum()),
                  'what': 'every answer of one step (batch 0): |D - D64| / D64, D64 recomputed in FP64 '
                          'from the raw samples (tm_result_fp64)'}

    # the plain FP32 kernel on the same batches and windows: the metric's own comparison
    plain = None
    if kname == 'k_scan_umma' and not args.no_fp32:
        ctx.set_kernel(tb.KERNEL_FP32)
        fsteps = min(args.steps, 3)
        fbatches = [ctx.batch(reqs[i * per:(i + 1) * per]) for i in range(min(nbatch, fsteps))]
        fbatches[0].run()  # warm-up
        ctx.profile_enable(True)
        ctx.profile_read()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        fpairs = 0
        for s in range(fsteps):
            fbatches[s % len(fbatches)].run()
            fpairs += pair_count[s % len(fbatches)]
        f1.record(stream)
        barrier()
        f_ms = f0.elapsed_time(f1)
        fk, fl, fkms, fkflops, _ = ctx.profile_read()
        ctx.profile_enable(False)
        for b in fbatches:
            b.close()
        ctx.set_kernel(kernel)
        plain = {'pairs': fpairs, 'ms': f_ms, 'kernel': fk, 'launches': fl, 'kernel_ms': fkms, 'flops': fkflops,
                 'steps': fsteps}

    from tremor_b200.replicas import combine
    dev = f'cuda:{local}'
    total_pairs, ms = combine(pairs, ms, dist, dev)  # every replica's pairs, the slowest rank's time
    _, e_ms = combine(0.0, e_ms, dist, dev)
    _, k_avg_ms = combine(0.0, kms / max(launches, 1), dist, dev)
    value = total_pairs / (ms / 1e3) / 1e9
    e2e_value = total_pairs / (e_ms / 1e3) / 1e9

    plain_line = None
    if plain is not None:
        fp_pairs, fp_ms = combine(plain['pairs'], plain['ms'], dist, dev)
        _, fk_avg = combine(0.0, plain['kernel_ms'] / max(plain['launches'], 1), dist, dev)
        plain_line = {'value': fp_pairs / (fp_ms / 1e3) / 1e9, 'unit': UNIT, 'steps': plain['steps'],
                      'ms_per_step': fp_ms / plain['steps'], 'kernel': plain['kernel'],
                      'kernel_ms_per_launch': fk_avg,
                      'what': 'the plain FP32 kernel (TM_KERNEL_FP32) on the same batches, after the split-BF16 '
                              'legs; CUDA events on the library stream'}
        try:
            fpk = tb.fp32_peak(local)
            ach = plain['flops'] / max(plain['launches'], 1) / (fk_avg / 1e3) / 1e12
            plain_line['roofline'] = {'bound': 'fp32', 'achieved': ach, 'peak': fpk, 'unit': 'TFLOP/s',
                                      'frac': ach / fpk,
                                      'peak_note': 'measured FP32 FMA rate (tm_fp32_peak)'}
        except Exception as exc:  # informative
            plain_line['roofline'] = {'error': str(exc)[:200]}

    if rank == 0:
        bf16_peak, _, peak_kind = peaks()
        flops_per_launch = kflops / max(launches, 1)
        achieved = flops_per_launch / (k_avg_ms / 1e3) / 1e12
        if kname == 'k_scan_umma':
            roof = {'bound': 'tensor', 'achieved': achieved, 'peak': bf16_peak / 3.0, 'unit': 'TFLOP/s',
                    'peak_note': f'{peak_kind} bf16 dense / 3 (three BF16 products per FP32 multiply-add)'}
        elif kname == 'fft':
            # the FFT branch (tm_fftk.cu): algorithmic bytes per launch = the piece spectra (16 B
            # per sample), the prefix sums (16 B), the raw sample and its constant run (6 B)
            _, hbm_peak, hbm_kind = peaks()
            fbytes = 38.0 * w['n']
            gbs = fbytes / (k_avg_ms / 1e3) / 1e9
            roof = {'bound': 'hbm', 'achieved': gbs, 'peak': hbm_peak, 'unit': 'GB/s',
                    'peak_note': f'{hbm_kind} HBM copy bandwidth; algorithmic bytes 38 B per sample per launch '
                                 '(spectra, prefix sums, raw, runs); the direct-contraction-equivalent rate is '
                                 'in direct_equivalent_tflops',
                    'algorithmic_bytes_per_launch': fbytes, 'direct_equivalent_tflops': achieved}
            achieved = gbs
        else:
            try:
                measured = tb.fp32_peak(local)
                roof = {'bound': 'fp32', 'achieved': achieved, 'peak': measured, 'unit': 'TFLOP/s',
                        'peak_note': 'measured FP32 FMA rate (tm_fp32_peak: register FMA chains on every SM)',
                        'peak_nominal': 148 * 128 * 2 * 1.965e9 / 1e12}
            except Exception:
                nominal = 148 * 128 * 2 * 1.965e9 / 1e12
                roof = {'bound': 'fp32', 'achieved': achieved, 'peak': nominal, 'unit': 'TFLOP/s',
                        'peak_note': 'nominal FP32 FMA peak (148 SMs x 128 lanes x 2 x 1.965 GHz)'}
        roof['frac'] = achieved / roof['peak']
        if kname == 'k_scan_umma':
            sustained = peaks_sustained()
            if sustained and k_avg_ms * args.steps >= 1000.0:
                # the kernel runs back to back for seconds under the power cap: the measured
                # sustained GEMM loop is its denominator; the burst figure stays beside it
                roof['peak_burst'], roof['frac_burst'] = roof['peak'], roof['frac']
                roof['peak'] = sustained / 3.0
                roof['frac'] = achieved / roof['peak']
                roof['peak_note'] = ('measured sustained bf16 dense / 3 (a seconds-long GEMM loop under the '
                                     'power cap; three BF16 products per FP32 multiply-add); the burst figure '
                                     'is in peak_burst')
        tb_bytes = traffic_for(kname, args.workload)
        roof['traffic'] = tb_bytes
        roof['kernel'] = kname
        roof['algorithmic_flops_per_launch'] = flops_per_launch
        roof['kernel_ms_per_launch'] = k_avg_ms
        cpu_v, cpu_info = (None, {'error': 'skipped'}) if args.no_cpu else cpu_reference(w, x, q)
        if not args.no_cpu:
            try:
                mv, minfo = cpu_mass(w, x, q)
                cpu_info['mass_v3'] = {'value': mv, 'unit': UNIT, **minfo}
            except Exception as exc:  # the MASS leg is informative; the reference scan is the baseline
                cpu_info['mass_v3'] = {'error': str(exc)[:200]}
        line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': ms / args.steps, 'higher_is_better': True, 'scaling': 'weak',
                'vs_baseline': value / plain_line['value'] if plain_line else None,
                'vs_baseline_note': 'value / plain_fp32.value: the metric is pairs/s against the plain FP32 '
                                    'kernel, measured in this run (no published number exists)'
                                    if plain_line else 'no FP32 leg in this run',
                'plain_fp32': plain_line,
                'fp64_error': fp64_error,
                'dtype': 'bf16x3+f32' if kname == 'k_scan_umma' else 'f32',
                'data': 'synthetic',
                'config': {'workload': args.workload, 'n': w['n'], 'templates': w['q'], 'templates_per_step': per,
                           'm': w['m'], 'mode': w['mode'], 'k': w['k'], 'merge': w['merge'], 'corr': w['corr'],
                           'events': w['events'], 'seed': w['seed'], 'kernel': args.kernel, 'tiles': args.tiles,
                           'l2': 'inputs larger than L2 (waveform 4n bytes)', 'parallelism': f'replicas x{world}'},
                'roofline': roof,
                'cpu_baseline': {'value': cpu_v, 'unit': UNIT, **cpu_info},
                'e2e': {'value': e2e_value, 'unit': UNIT, 'h2d_bytes_per_step': h2d // args.steps,
                        'd2h_bytes_per_step': d2h // args.steps},
                'gpu_launches': all_launches, 'clocks': clocks,
                'd2h_bytes_per_step_value': d2h_value // args.steps,
                'candidates_last_step': ctx.last_candidates(),
                'phases_ms_per_step': phase_ms,
                'step_ms': [round(a.elapsed_time(b), 3) for a, b in zip(step_ev, step_ev[1:])]}
    for b in batches:
        b.close()
    ctx.close()
    if rank == 0:
        if w.get('serving_leg') and world == 1 and not args.no_serving:
            try:
                line['serving'] = serving_leg(local, batch_ms=args.batch_ms)
            except Exception as exc:  # an informative leg
                line['serving'] = {'error': str(exc)[:300]}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=5)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', choices=['ours', 'reference'], default='ours')
    p.add_argument('--workload', choices=sorted(WORKLOADS), default='precision')
    p.add_argument('--kernel', choices=['auto', 'fp32', 'bf16'], default=None,
                   help='contraction kernel (default: the workload\'s, else auto)')
    p.add_argument('--tiles', choices=['auto', 'rows', 'cols128', 'cols64', 'cols32'], default='auto',
                   help='tile shape of mixed-length groups (TILES_*)')
    p.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline leg')
    p.add_argument('--no-fp32', action='store_true', help='skip the plain FP32 kernel leg')
    p.add_argument('--no-serving', action='store_true', help='skip the short serving leg of the default workload')
    p.add_argument('--rate', type=float, default=0.0, help='serving: Poisson arrival rate (req/s)')
    p.add_argument('--requests', type=int, default=0, help='serving: requests in the timed stream')
    p.add_argument('--workers', type=int, default=1, help='serving: batches in flight at once')
    p.add_argument('--max-batch', type=int, default=256, help='serving: requests per batch at most')
    p.add_argument('--batch-ms', type=float, default=0.0, help='serving: modelled device ms per batch at most (0: none)')
    args = p.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    w = WORKLOADS[args.workload]
    if args.impl == 'reference':
        run_reference(args, w)
    elif w.get('serve'):
        run_serving(args, w)
    else:
        run_ours(args, w)


if __name__ == '__main__':
    main()
