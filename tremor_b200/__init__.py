"""tremor_b200 — TREMOR's exact template-matching scan on one B200.

Python binding of the C ABI in include/tremor_b200.h (libtremor_b200.so, built by
``python -m tremor_b200.build``). The search calls mirror the reference's
``SkipSequentialScan`` (tremor/algos/sss/SkipSequential.hpp:32-78):

    ctx = Context(waveform)                       # ~ SkipSequentialScan::build
    I, D = ctx.search_knn(queries, k, merge)      # ~ search_knn (Tremor::searchIndex I/D)
    hits = ctx.search_threshold(queries, 0.8, 0)  # ~ search_threshold
    rows = knn_rows(I, D, m)                      # the reference's CSV rows

There is no CPU fallback: without the native library or a CUDA device every call
raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path
from typing import List, Sequence, Tuple

import numpy as np

__all__ = ['Context', 'Batch', 'TremorError', 'Request', 'knn_rows', 'threshold_rows', 'load_library',
           'MODE_KNN', 'MODE_THRESHOLD', 'KERNEL_AUTO', 'KERNEL_FP32', 'KERNEL_SPLIT_BF16', 'MISSING_VALUE']

MODE_THRESHOLD = 0
MODE_KNN = 1
KERNEL_AUTO, KERNEL_FP32, KERNEL_SPLIT_BF16 = 0, 1, 2
TILES_AUTO, TILES_ROWS, TILES_COLS_128, TILES_COLS_64, TILES_COLS_32, TILES_FFT = 0, 1, 2, 3, 4, 5
FLAG_ZNORMALIZED = 1
MISSING_VALUE = np.float32(-100000.0)
FLT_MAX = float(np.finfo(np.float32).max)

_ERRORS = {-1: 'invalid argument', -2: 'CUDA error', -3: 'out of memory', -4: 'invalid state',
           -5: 'buffer too small', -6: 'no usable sm_100 device', -7: 'kernel wait timed out'}

LIB_PATH = Path(__file__).resolve().parent / 'libtremor_b200.so'
_lib = None
_vp = ctypes.c_void_p


class TremorError(RuntimeError):
    def __init__(self, code: int, detail: str = ''):
        super().__init__(f'{_ERRORS.get(code, "error")} ({code}){": " + detail if detail else ""}')
        self.code = code


class _Request(ctypes.Structure):
    _fields_ = [('templ', _vp), ('m', ctypes.c_int32), ('mode', ctypes.c_int32), ('k', ctypes.c_int32),
                ('merge_offset', ctypes.c_int32), ('correlation', ctypes.c_float), ('flags', ctypes.c_uint32)]


class _ServeConfig(ctypes.Structure):
    _fields_ = [('workers', ctypes.c_int32), ('max_batch', ctypes.c_int32), ('memory_budget', ctypes.c_uint64),
                ('batch_ms', ctypes.c_double)]


class _Completion(ctypes.Structure):
    _fields_ = [('ticket', ctypes.c_uint64), ('status', ctypes.c_int32), ('batch_size', ctypes.c_int32),
                ('result', _vp), ('submit_ms', ctypes.c_double), ('start_ms', ctypes.c_double),
                ('done_ms', ctypes.c_double)]


def load_library():
    """Loads libtremor_b200.so; raises ImportError when it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f'{LIB_PATH} is missing: build it with `python -m tremor_b200.build`')
    lib = ctypes.CDLL(str(LIB_PATH))
    i, u64, f, pp = ctypes.c_int, ctypes.c_uint64, ctypes.c_float, ctypes.POINTER(_vp)
    sig = {
        'tm_ctx_create': (i, [_vp, u64, i, pp]),
        'tm_ctx_destroy': (i, [_vp]),
        'tm_last_error': (ctypes.c_char_p, [_vp]),
        'tm_set_kernel': (i, [_vp, i]),
        'tm_set_tiles': (i, [_vp, i]),
        'tm_autotune': (i, [_vp, _vp, i]),
        'tm_set_tile_model': (i, [_vp, _vp, i]),
        'tm_set_window_range': (i, [_vp, u64, u64]),
        'tm_prepare_length': (i, [_vp, i]),
        'tm_window_stats': (i, [_vp, i, u64, u64, _vp, _vp]),
        'tm_search_knn': (i, [_vp, _vp, i, i, i, i, _vp, _vp]),
        'tm_search_threshold': (i, [_vp, _vp, i, i, f, i, pp]),
        'tm_scan_batch': (i, [_vp, _vp, i, pp]),
        'tm_result_count': (i, [_vp, i, ctypes.POINTER(u64)]),
        'tm_result_get': (i, [_vp, i, _vp, _vp, u64]),
        'tm_result_free': (None, [_vp]),
        'tm_result_fp64': (i, [_vp, _vp, i, _vp, i, _vp, u64]),
        'tm_cc_to_ed': (f, [f, i]),
        'tm_ed_to_cc': (f, [f, i]),
        'tm_profile_enable': (i, [_vp, i]),
        'tm_profile_read': (i, [_vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64),
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(ctypes.c_int64)]),
        'tm_profile_phases': (i, [_vp, _vp, i]),
        'tm_scan_knn': (i, [_vp, _vp, i, i, i, f, _vp, _vp]),
        'tm_fp32_peak': (i, [i, ctypes.POINTER(ctypes.c_double)]),
        'tm_scan_threshold': (i, [_vp, _vp, i, f, i, pp]),
        'tm_serve_start': (i, [_vp, _vp]),
        'tm_submit': (i, [_vp, _vp, ctypes.POINTER(u64)]),
        'tm_poll': (i, [_vp, _vp, i, i, ctypes.POINTER(i)]),
        'tm_serve_stop': (i, [_vp]),
        'tm_serve_status': (i, [_vp, ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u64),
                                ctypes.POINTER(u64)]),
        'tm_last_candidates': (i, [_vp, ctypes.POINTER(u64)]),
        'tm_batch_create': (i, [_vp, _vp, i, pp]),
        'tm_batch_run': (i, [_vp, _vp, pp]),
        'tm_batch_destroy': (i, [_vp]),
        'tm_batch_h2d_bytes': (i, [_vp, ctypes.POINTER(u64)]),
        'tm_d2h_bytes': (i, [_vp, ctypes.POINTER(u64)]),
        'tm_ctx_stream': (i, [_vp, pp]),
        'tm_bound_diagnostics': (i, [_vp, _vp, i, i, _vp, _vp, _vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


class Request:
    """One template request (kNN or threshold), as tm_request."""

    def __init__(self, template, mode=MODE_KNN, k=1, merge_offset=0, correlation=0.0, znormalized=False):
        self.template = np.ascontiguousarray(template, dtype=np.float32)
        self.mode, self.k, self.merge_offset = int(mode), int(k), int(merge_offset)
        self.correlation = float(correlation)
        self.flags = FLAG_ZNORMALIZED if znormalized else 0


class Context:
    """A waveform resident on one GPU (tm_ctx)."""

    def __init__(self, waveform: np.ndarray, device: int = 0):
        self._lib = load_library()
        self.waveform = np.ascontiguousarray(waveform, dtype=np.float32)
        self.n = len(self.waveform)
        h = _vp()
        rc = self._lib.tm_ctx_create(_ptr(self.waveform), self.n, device, ctypes.byref(h))
        if rc != 0:
            raise TremorError(rc, 'tm_ctx_create')
        self._h = h

    def close(self):
        if getattr(self, '_h', None):
            self._lib.tm_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise TremorError(rc, self._lib.tm_last_error(self._h).decode())

    @staticmethod
    def relative_error(dist: np.ndarray, fp64: np.ndarray) -> np.ndarray:
        """|D - D64| / D64 per answer (NaN for padding and constant windows, whose FP64
        distance is +inf)."""
        d = np.asarray(dist, np.float64)
        f = np.asarray(fp64, np.float64)
        with np.errstate(divide='ignore', invalid='ignore'):
            return np.where(np.isfinite(f), np.abs(d - f) / f, np.nan)

    def set_kernel(self, kernel: int):
        self._check(self._lib.tm_set_kernel(self._h, kernel))

    def set_tiles(self, tiles: int):
        """Tile shape of mixed-length groups (TILES_*), for batches created afterwards."""
        self._check(self._lib.tm_set_tiles(self._h, tiles))

    def autotune(self):
        """Measures the planner's model on this device (tm_autotune): (table, fft_ms,
        fft_long_ms). table: milliseconds of 128 templates x 2^25 windows, shape [kind (one
        length, several), tile shape (rows, columns 128 / 64 / 32), K (256, 1024, 4096,
        16384)]; fft_ms, fft_long_ms: the FFT branch's milliseconds per template per 2^25
        samples for templates of up to 8192 samples and for longer ones."""
        out = np.zeros(34, np.float64)
        rc = self._lib.tm_autotune(self._h, out.ctypes.data, 34)
        self._check(min(rc, 0))
        return out[:32].reshape(2, 4, 4), float(out[32]), float(out[33])

    def set_tile_model(self, ms: np.ndarray, fft_ms: float = None, fft_long_ms: float = None):
        arr = np.ascontiguousarray(ms, dtype=np.float64).reshape(-1)
        if fft_ms is not None:
            arr = np.concatenate([arr, [float(fft_ms)]])
            if fft_long_ms is not None:
                arr = np.concatenate([arr, [float(fft_long_ms)]])
        self._check(self._lib.tm_set_tile_model(self._h, arr.ctypes.data, len(arr)))

    def set_window_range(self, first: int, count: int):
        self._check(self._lib.tm_set_window_range(self._h, first, count))

    def prepare_length(self, m: int):
        self._check(self._lib.tm_prepare_length(self._h, m))

    def window_stats(self, m: int, first: int = 0, count: int | None = None):
        """The reference's per-window (mean, std) floats (SkipSequential.cpp:157-190)."""
        if count is None:
            count = self.n - m + 1 - first
        mean = np.zeros(count, np.float32)
        std = np.zeros(count, np.float32)
        self._check(self._lib.tm_window_stats(self._h, m, first, count, _ptr(mean), _ptr(std)))
        return mean, std

    def search_knn(self, queries: np.ndarray, k: int, merge_offset: int = 0) -> Tuple[np.ndarray, np.ndarray]:
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        I = np.zeros((q.shape[0], k), np.uint64)
        D = np.zeros((q.shape[0], k), np.float32)
        self._check(self._lib.tm_search_knn(self._h, _ptr(q), q.shape[0], q.shape[1], k, merge_offset,
                                            _ptr(I), _ptr(D)))
        return I, D

    def search_threshold(self, queries: np.ndarray, correlation: float, merge_offset: int = 0):
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        res = _vp()
        self._check(self._lib.tm_search_threshold(self._h, _ptr(q), q.shape[0], q.shape[1], correlation,
                                                  merge_offset, ctypes.byref(res)))
        return self._take(res, q.shape[0])

    @staticmethod
    def _requests(requests: Sequence[Request]):
        arr = (_Request * len(requests))()
        for i, r in enumerate(requests):
            arr[i] = _Request(_ptr(r.template), len(r.template), r.mode, r.k, r.merge_offset, r.correlation,
                              r.flags)
        return arr

    def scan_batch(self, requests: Sequence[Request], fp64: bool = False):
        """Answers (positions, distances) per request, any mix of modes and lengths. With
        fp64=True each request's answers are (positions, distances, fp64_distances): every
        answer's distance recomputed entirely in FP64 (tm_result_fp64), so its error
        against FP64 is stated per result."""
        arr = self._requests(requests)
        res = _vp()
        self._check(self._lib.tm_scan_batch(self._h, arr, len(requests), ctypes.byref(res)))
        return self._take(res, len(requests), requests if fp64 else None)

    def serve(self, workers: int = 1, max_batch: int = 256, memory_budget: int = 0, batch_ms: float = 0.0) -> 'Server':
        """Starts continuous batching over this context's waveform (tm_serve_start); batch_ms
        bounds a batch's modelled device time (0: no bound)."""
        return Server(self, workers, max_batch, memory_budget, batch_ms)

    def scan_knn(self, template: np.ndarray, k: int, merge_offset: int = 0, bound: float = float('inf')):
        """(positions, distances) of one template's k answers (tm_scan_knn); answers above
        `bound` come back as (0, FLT_MAX)."""
        q = np.ascontiguousarray(template, dtype=np.float32)
        pos = np.zeros(k, np.uint64)
        dist = np.zeros(k, np.float32)
        b = float(np.finfo(np.float32).max) if not np.isfinite(bound) else float(bound)
        self._check(self._lib.tm_scan_knn(self._h, _ptr(q), len(q), k, merge_offset, b, _ptr(pos), _ptr(dist)))
        return pos, dist

    def scan_threshold(self, template: np.ndarray, correlation: float, merge_offset: int = 0):
        """(positions, distances) of one template's threshold hits (tm_scan_threshold)."""
        q = np.ascontiguousarray(template, dtype=np.float32)
        res = _vp()
        self._check(self._lib.tm_scan_threshold(self._h, _ptr(q), len(q), float(correlation), merge_offset,
                                                ctypes.byref(res)))
        return self._take(res, 1)[0]

    def batch(self, requests: Sequence[Request]) -> 'Batch':
        """A prepared batch whose templates stay resident on the device (tm_batch)."""
        return Batch(self, requests)

    def stream(self) -> int:
        """The context's cudaStream_t as an integer handle."""
        s = _vp()
        self._check(self._lib.tm_ctx_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def d2h_bytes(self) -> int:
        n = ctypes.c_uint64(0)
        self._check(self._lib.tm_d2h_bytes(self._h, ctypes.byref(n)))
        return n.value

    def _take(self, res, count, fp64_requests=None) -> List[Tuple[np.ndarray, ...]]:
        """Copies the answers out of a tm_result and frees it. With fp64_requests (the
        requests of the result, in order), each entry also carries the FP64 distances of its
        answers (tm_result_fp64)."""
        out = []
        try:
            for i in range(count):
                n = ctypes.c_uint64(0)
                self._check(self._lib.tm_result_count(res, i, ctypes.byref(n)))
                pos = np.zeros(n.value, np.uint64)
                dist = np.zeros(n.value, np.float32)
                self._check(self._lib.tm_result_get(res, i, _ptr(pos), _ptr(dist), n.value))
                if fp64_requests is None:
                    out.append((pos, dist))
                    continue
                t = fp64_requests[i].template
                d64 = np.zeros(n.value, np.float64)
                self._check(self._lib.tm_result_fp64(self._h, res, i, _ptr(t), len(t), _ptr(d64), n.value))
                out.append((pos, dist, d64))
        finally:
            self._lib.tm_result_free(res)
        return out

    def profile_enable(self, on: bool = True):
        self._check(self._lib.tm_profile_enable(self._h, 1 if on else 0))

    def profile_read(self):
        """(kernel name, launches, device ms, algorithmic flops, all library launches); resets."""
        name = ctypes.create_string_buffer(64)
        launches, allk = ctypes.c_int64(0), ctypes.c_int64(0)
        ms, flops = ctypes.c_double(0), ctypes.c_double(0)
        self._check(self._lib.tm_profile_read(self._h, name, 64, ctypes.byref(launches), ctypes.byref(ms),
                                              ctypes.byref(flops), ctypes.byref(allk)))
        return name.value.decode(), launches.value, ms.value, flops.value, allk.value

    PHASES = ('contraction', 'bound_list_repass', 'rescore', 'answer_sort', 'copy_back', 'host_answers')

    def profile_phases(self):
        """{phase: milliseconds} spent in each phase of the searches since the last call,
        while profiling was enabled (tm_profile_phases); resets."""
        out = np.zeros(8, dtype=np.float64)
        n = self._lib.tm_profile_phases(self._h, out.ctypes.data, len(out))
        self._check(min(n, 0))
        return dict(zip(self.PHASES, out[:n].tolist()))

    def bound_diagnostics(self, queries: np.ndarray, exact: bool = True):
        """(d, e, exact) arrays [templates, windows]: the contraction kernel's distance, its
        error bound, and the reference's exact distance of every pair (tm_bound_diagnostics)."""
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        m = q.shape[1]
        W = self.n - m + 1
        d = np.zeros((q.shape[0], W), np.float32)
        e = np.zeros((q.shape[0], W), np.float32)
        x = np.zeros((q.shape[0], W), np.float32) if exact else None
        self._check(self._lib.tm_bound_diagnostics(self._h, _ptr(q), q.shape[0], m, _ptr(d), _ptr(e),
                                                   _ptr(x) if exact else None))
        return d, e, x

    def last_candidates(self) -> int:
        n = ctypes.c_uint64(0)
        self._check(self._lib.tm_last_candidates(self._h, ctypes.byref(n)))
        return n.value


class Batch:
    """Requests prepared once and resident on the device; run() any number of times."""

    def __init__(self, ctx: Context, requests: Sequence[Request]):
        self.ctx, self.count = ctx, len(requests)
        self._keep = list(requests)
        arr = ctx._requests(requests)
        h = _vp()
        ctx._check(ctx._lib.tm_batch_create(ctx._h, arr, len(requests), ctypes.byref(h)))
        self._h = h

    def run(self, fp64: bool = False):
        """Answers per request; with fp64=True also each answer's FP64 distance (as
        Context.scan_batch)."""
        res = _vp()
        self.ctx._check(self.ctx._lib.tm_batch_run(self.ctx._h, self._h, ctypes.byref(res)))
        return self.ctx._take(res, self.count, self._keep if fp64 else None)

    def h2d_bytes(self) -> int:
        n = ctypes.c_uint64(0)
        self.ctx._check(self.ctx._lib.tm_batch_h2d_bytes(self._h, ctypes.byref(n)))
        return n.value

    def close(self):
        if getattr(self, '_h', None):
            self.ctx._lib.tm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Completion:
    """One served request: its ticket, status (0 = answers present), answers (positions,
    distances) and times in ms since the server started (submitted, batch admitted,
    done), with the size of the batch that carried it."""

    def __init__(self, ticket, status, answers, submit_ms, start_ms, done_ms, batch_size):
        self.ticket, self.status, self.answers = ticket, status, answers
        self.submit_ms, self.start_ms, self.done_ms, self.batch_size = submit_ms, start_ms, done_ms, batch_size

    @property
    def latency_ms(self) -> float:
        return self.done_ms - self.submit_ms


class Server:
    """Continuous batching over a context's resident waveform (tm_serve_*): submit() from
    any thread, poll() from one."""

    def __init__(self, ctx: Context, workers: int = 1, max_batch: int = 256, memory_budget: int = 0,
                 batch_ms: float = 0.0):
        self.ctx = ctx
        cfg = _ServeConfig(workers, max_batch, memory_budget, batch_ms)
        ctx._check(ctx._lib.tm_serve_start(ctx._h, ctypes.byref(cfg)))
        self._running = True

    def submit(self, request: Request) -> int:
        arr = Context._requests([request])
        t = ctypes.c_uint64(0)
        self.ctx._check(self.ctx._lib.tm_submit(self.ctx._h, arr, ctypes.byref(t)))
        return t.value

    def poll(self, max_count: int = 256, timeout_ms: int = 100) -> List[Completion]:
        buf = (_Completion * max_count)()
        n = ctypes.c_int(0)
        self.ctx._check(self.ctx._lib.tm_poll(self.ctx._h, buf, max_count, int(timeout_ms), ctypes.byref(n)))
        out = []
        for c in buf[:n.value]:
            answers = self.ctx._take(_vp(c.result), 1)[0] if c.status == 0 and c.result else None
            out.append(Completion(c.ticket, c.status, answers, c.submit_ms, c.start_ms, c.done_ms, c.batch_size))
        return out

    def status(self):
        """(requests pending, requests in flight, admitted device bytes in flight, kernel
        launches of the served batches so far)."""
        a, b, c, d = (ctypes.c_uint64(0) for _ in range(4))
        self.ctx._check(self.ctx._lib.tm_serve_status(self.ctx._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                                      ctypes.byref(d)))
        return a.value, b.value, c.value, d.value

    def stop(self):
        """Completes everything submitted; completions stay pollable."""
        if self._running:
            self._running = False
            self.ctx._check(self.ctx._lib.tm_serve_stop(self.ctx._h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()


def fp32_peak(device: int = 0) -> float:
    """Measured FP32 FMA rate of the device in TFLOP/s (tm_fp32_peak)."""
    lib = load_library()
    v = ctypes.c_double(0.0)
    rc = lib.tm_fp32_peak(device, ctypes.byref(v))
    if rc != 0:
        raise TremorError(rc, 'tm_fp32_peak')
    return v.value


def ed_to_cc(ed: float, m: int) -> float:
    return load_library().tm_ed_to_cc(float(ed), m)


def knn_rows(I: np.ndarray, D: np.ndarray, m: int):
    """kNN answers as the reference's writer prints them: tID, k, pos, corr (SkipSequential.cpp:461-470)."""
    lib = load_library()
    return [[str(q), str(j + 1), str(int(I[q, j])), '%f' % lib.tm_ed_to_cc(float(D[q, j]), m)]
            for q in range(I.shape[0]) for j in range(I.shape[1])]


def threshold_rows(hits, m: int):
    """Threshold hits as the reference's writer prints them: Query, Counter, Position, Cross Correlation."""
    lib = load_library()
    rows = []
    for q, (pos, dist) in enumerate(hits):
        for c, (p, d) in enumerate(zip(pos, dist)):
            rows.append([str(q), str(c), str(int(p)), '%f' % lib.tm_ed_to_cc(float(d), m)])
    return rows
