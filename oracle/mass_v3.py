"""MASS V3 on the CPU: a restatement of the reference's distributed-MASS baseline
(dmass/DMASS_V3.c) for one rank. TEST AND BASELINE INFRASTRUCTURE: bench.py times it
as the CPU MASS baseline and tests/test_oracle.py checks it; the GPU product never
uses it.

FFTW 3 (the reference's FFT, `fftw/3.3.9` in experiments/validate_search.slurm:13) is
not installed here, so the FFTs are scipy.fft's pocketfft (double precision r2c/c2r,
`workers` threads), which computes the same transforms.

  MassV3(x, m)           mass_ctx_init (DMASS_V3.c:798-887): pieces of fft_len points
                         (2^15, doubled until >= 4m) overlapping by m - 1 (overlap-save),
                         their spectra, exact two-pass window statistics, fft_dot_min
  MassV3.distances(y)    mass_ctx_query (DMASS_V3.c:904-996): z-normalised query
                         (zNorm, :998), reversed-query spectrum, one c2r per piece, the
                         sliding dot products, Pearson -> ED^2 = 2m(1 - c) clamped, direct
                         dot products for windows with m*sigma < fft_dot_min; FLT_MAX for
                         missing or constant windows
"""
from __future__ import annotations

import os

import numpy as np

MISSING = np.float32(-100000.0)
FLT_MAX = float(np.finfo(np.float32).max)


class MassV3:
    def __init__(self, x: np.ndarray, m: int, workers: int | None = None):
        import scipy.fft as sfft
        self.fft = sfft
        self.workers = workers or os.cpu_count() or 1
        raw = np.asarray(x, dtype=np.float32)
        self.missing = raw == MISSING
        self.x = np.where(self.missing, 0.0, raw.astype(np.float64))  # load_data :653, missing -> 0 in use
        n = len(raw)
        self.n, self.m = n, m
        L = 1 << 15
        while L < 4 * m:
            L *= 2
        self.L = L
        self.W = n - m + 1
        self.step = L - m + 1
        self.pieces = (self.W + self.step - 1) // self.step
        starts = np.arange(self.pieces) * self.step
        idx = starts[:, None] + np.arange(L)[None, :]
        blocks = np.where(idx < n, self.x[np.minimum(idx, n - 1)], 0.0)
        self.X = sfft.rfft(blocks, axis=1, workers=self.workers)
        if self.W * m <= (1 << 26):
            # exact two-pass statistics (:854-873)
            win = np.lib.stride_tricks.sliding_window_view(self.x, m)
            self.mu = win.mean(axis=1)
            self.sigma = np.sqrt(((win - self.mu[:, None]) ** 2).mean(axis=1))
        else:
            # large inputs (baseline timing only; the statistics are not timed): FP64 prefix
            # sums of the centred waveform instead of numpy two-pass over W x m samples
            c = self.x - self.x.mean()
            p1 = np.concatenate(([0.0], np.cumsum(c)))
            p2 = np.concatenate(([0.0], np.cumsum(c * c)))
            s1 = p1[m:] - p1[:-m]
            s2 = p2[m:] - p2[:-m]
            mu_c = s1 / m
            self.mu = mu_c + self.x.mean()
            self.sigma = np.sqrt(np.maximum(s2 / m - mu_c * mu_c, 0.0))
        sumsq = float(np.sum(self.x * self.x))
        self.fft_dot_min = 1e4 * np.finfo(np.float64).eps * np.log2(L) * np.sqrt(sumsq) * np.sqrt(m)

    def distances(self, y: np.ndarray) -> np.ndarray:
        m, L = self.m, self.L
        y = np.asarray(y, dtype=np.float64)
        ex, ex2 = y.sum(), (y * y).sum()
        mean = ex / m
        y = (y - mean) / np.sqrt(ex2 / m - mean * mean)  # zNorm (:998-1011)
        meany = y.sum() / m
        sigmay = np.sqrt(max((y * y).sum() / m - meany * meany, 0.0))
        if not np.isfinite(sigmay) or sigmay <= 1e-12:
            return np.full(self.W, FLT_MAX)
        yb = np.zeros(L)
        yb[:m] = y[::-1]
        Y = self.fft.rfft(yb, workers=self.workers)
        dots = self.fft.irfft(self.X * Y[None, :], n=L, axis=1, workers=self.workers)
        buf = dots[:, m - 1:m - 1 + self.step].reshape(-1)[: self.W]
        sumxy = buf.copy()
        low = np.flatnonzero(m * self.sigma < self.fft_dot_min)
        if len(low):
            win = np.lib.stride_tricks.sliding_window_view(self.x, m)
            sumxy[low] = win[low] @ y
        with np.errstate(invalid='ignore', divide='ignore'):
            c = (sumxy - m * self.mu * meany) / (m * self.sigma * sigmay)
        c = np.clip(c, -1.0, 1.0)
        d = 2 * m * (1 - c)
        bad = self.missing[: self.W] | ~np.isfinite(self.sigma) | (self.sigma <= 1e-12)
        d[bad] = FLT_MAX
        return d
