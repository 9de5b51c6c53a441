"""Measures the tile-shape model of the tensor-core contraction on this GPU and prints it
(or saves it as JSON for Context.set_tile_model):

    python -m tremor_b200.autotune [--out model.json]

The model is the kernel time in milliseconds of 128 templates against 2^25 windows, per
group kind (one length; several lengths, measured with 128 distinct lengths K - 127 .. K,
as batches of lengths drawn from a continuous range have), tile shape (128-template row
tiles; window-major column tiles of 128, 64 and 32 templates) and template length K;
TILES_AUTO picks the shape (or the FFT branch, whose per-template time is measured too,
on templates of distinct lengths) of least modelled time from it."""
from __future__ import annotations

import argparse
import json

import numpy as np

import tremor_b200 as tb

SHAPES = ('rows (k_scan_umma)', 'columns 128 (k_scan_wm)', 'columns 64 (k_scan_wm)', 'columns 32 (k_scan_wm)')
KS = (256, 1024, 4096, 16384)


def main():
    p = argparse.ArgumentParser()
    p.add_argument('--out', help='write the model as JSON')
    p.add_argument('--device', type=int, default=0)
    args = p.parse_args()
    with tb.Context(np.random.default_rng(0).normal(size=1 << 16).astype(np.float32), device=args.device) as ctx:
        table, fft_ms, fft_long_ms = ctx.autotune()
    for kind, name in enumerate(('one length', 'several lengths')):
        print(f'{name}: ms per 128 templates x 2^25 windows, K = {KS}')
        for v, shape in enumerate(SHAPES):
            tf = [2.0 * 128 * (1 << 25) * k / (table[kind, v, i] * 1e-3) / 1e12 for i, k in enumerate(KS)]
            print(f'  {shape:26s} ' + '  '.join(f'{table[kind, v, i]:8.1f} ms ({t:5.0f} TF)' for i, t in
                                                  enumerate(tf)))
    print(f'FFT branch: {fft_ms:.3f} ms per template per 2^25 samples (lengths up to 8192), '
          f'{fft_long_ms:.3f} (8193 to 16384)')
    if args.out:
        with open(args.out, 'w') as f:
            json.dump({'k': KS, 'shapes': SHAPES, 'ms': table.tolist(), 'fft_ms': fft_ms,
                       'fft_long_ms': fft_long_ms}, f, indent=1)


if __name__ == '__main__':
    main()
