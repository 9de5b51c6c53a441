"""Seeded synthetic seismic waveforms and templates.

The reference's paper datasets (Maule, SeiFR; see the reference README) are not
available here, so every benchmark and parity case runs on this generator:

* waveform: AR(2) coloured Gaussian noise ``x_t = 1.6 x_{t-1} - 0.7 x_{t-2} + e_t``
  times a slow amplitude envelope ``exp(w)`` where ``w`` is a mean-reverting random
  walk on a coarse grid (one step per 4096 samples, linearly interpolated), so the
  amplitude drifts by a factor of a few over the record without blowing up;
* templates: Gaussian-windowed linear chirps of 2-20 cycles across the window plus
  10 % white noise (relative to the chirp's RMS);
* events: copies of the templates added at uniform random offsets with amplitude SNR
  uniform in [0.5, 3], the ratio of the event's RMS to the RMS of the waveform
  under it (so an event's own window correlates at roughly snr / sqrt(1 + snr^2)).

Everything is float32 little-endian, as the reference's binary waveform files.
"""
from __future__ import annotations

import numpy as np

MISSING_VALUE = np.float32(-100000.0)  # TREMOR_MISSING_VALUE, ZnormSearch.hpp:21


def chirp_templates(count: int, m: int, rng: np.random.Generator, center_freq: bool = False) -> np.ndarray:
    """`count` Gaussian-windowed linear chirps of length `m` (float32, count x m).

    With ``center_freq`` the chirp band is placed around a random centre frequency
    (the batching workload's "random centre frequency" templates)."""
    t = np.linspace(0.0, 1.0, m, endpoint=False)
    out = np.empty((count, m), dtype=np.float32)
    for i in range(count):
        if center_freq:
            fc = rng.uniform(3.0, 18.0)
            span = rng.uniform(0.5, 1.0) * min(fc - 2.0, 20.0 - fc)
            f0, f1 = fc - span, fc + span
        else:
            f0 = rng.uniform(2.0, 10.0)
            f1 = rng.uniform(f0, 20.0)
        phase = 2.0 * np.pi * (f0 * t + 0.5 * (f1 - f0) * t * t)
        env = np.exp(-0.5 * ((t - 0.5) / rng.uniform(0.15, 0.3)) ** 2)
        c = env * np.sin(phase + rng.uniform(0, 2 * np.pi))
        c += 0.1 * np.sqrt(np.mean(c * c)) * rng.normal(size=m)
        out[i] = c.astype(np.float32)
    return out


def ar2_waveform(n: int, rng: np.random.Generator, chunk: int = 1 << 24) -> np.ndarray:
    """AR(2) noise (1.6, -0.7) times a slow mean-reverting log-amplitude envelope."""
    from scipy.signal import lfilter

    out = np.empty(n, dtype=np.float32)
    zi = np.zeros(2)
    for s in range(0, n, chunk):
        e = rng.normal(size=min(chunk, n - s))
        y, zi = lfilter([1.0], [1.0, -1.6, 0.7], e, zi=zi)
        out[s:s + len(y)] = y
    grid = n // 4096 + 2
    w = np.empty(grid)
    w[0] = 0.0
    steps = rng.normal(scale=0.05, size=grid)
    for i in range(1, grid):  # grid is small (n / 4096)
        w[i] = 0.99 * w[i - 1] + steps[i]
    w -= np.median(w)
    for s in range(0, n, chunk):
        idx = np.arange(s, min(s + chunk, n))
        out[s:s + len(idx)] *= np.exp(np.interp(idx / 4096.0, np.arange(grid), w)).astype(np.float32)
    return out


def inject_events(x: np.ndarray, templates: np.ndarray, events: int, rng: np.random.Generator) -> np.ndarray:
    """Adds `events` copies of the templates (cycled) at uniform offsets; returns the offsets."""
    n = len(x)
    noise = float(np.std(x[: min(n, 1 << 20)]))
    offsets = np.sort(rng.integers(0, n - templates.shape[1], size=events))
    for e, off in enumerate(offsets):
        tpl = templates[e % len(templates)].astype(np.float64)
        tpl = tpl / (np.sqrt(np.mean(tpl * tpl)) + 1e-30)
        snr = rng.uniform(0.5, 3.0)
        local = np.std(x[off:off + templates.shape[1]]) or noise
        x[off:off + templates.shape[1]] += (snr * local * tpl).astype(np.float32)
    return offsets


def workload(n: int, q: int, m: int, events: int, seed: int, center_freq: bool = False):
    """(waveform float32[n], templates float32[q, m], event offsets)."""
    rng = np.random.default_rng(seed)
    templates = chirp_templates(q, m, rng, center_freq)
    x = ar2_waveform(n, rng)
    offsets = inject_events(x, templates, events, rng)
    return x, templates, offsets


def mixed_workload(n: int, q: int, m_lo: int, m_hi: int, events: int, seed: int):
    """(waveform, list of templates with lengths log-uniform in [m_lo, m_hi] rounded to
    multiples of 16, event offsets): the batching workload."""
    rng = np.random.default_rng(seed)
    lengths = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), size=q))
    lengths = np.clip((np.round(lengths / 16) * 16).astype(int), m_lo, m_hi)
    templates = [chirp_templates(1, int(m), rng, center_freq=True)[0] for m in lengths]
    x = ar2_waveform(n, rng)
    noise = float(np.std(x[: min(n, 1 << 20)]))
    offsets = np.sort(rng.integers(0, n - m_hi, size=events))
    for e, off in enumerate(offsets):
        tpl = templates[e % q].astype(np.float64)
        tpl = tpl / (np.sqrt(np.mean(tpl * tpl)) + 1e-30)
        snr = rng.uniform(0.5, 3.0)
        local = np.std(x[off:off + len(tpl)]) or noise
        x[off:off + len(tpl)] += (snr * local * tpl).astype(np.float32)
    return x, templates, offsets
