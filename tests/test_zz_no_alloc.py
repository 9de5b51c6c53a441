"""tm_window_stats_noalloc, the allocation-free statistics entry point.

It serves callers that must not allocate device memory: a live detector with a fixed
latency budget (cudaMalloc may synchronise the device), a runtime whose pool allocator
holds the free memory. They own the input and
output device buffers (here: torch tensors made by the test, not by the call).

Checked through the C ABI: two calls in a row (two template lengths, the second reusing
the shared fixed scratch), each against tm_window_stats, the allocating entry point,
within 2^-21 relative (a few float ulps; the two compute the same FP64 quantities in
different orders), with the constant-window and missing-first-sample classification
identical. This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest

import tremor_b200 as tb

pytestmark = pytest.mark.gpu

REL = 2.0 ** -21


def _waveform(n, seed):
    rng = np.random.default_rng(seed)
    x = (rng.normal(size=n) * 2.0 + 0.5).astype(np.float32)
    x[1000:3000] = 4.0                              # constant windows
    x[50000:52000] *= np.float32(1e5)               # loud
    x[52000:60000] *= np.float32(1e-4)              # quiet after loud
    x[rng.integers(0, n, 40)] = tb.MISSING_VALUE    # scattered missing samples
    x[80000:80300] = tb.MISSING_VALUE               # a gap
    return x


def test_noalloc_stats_equal_allocating_entry_point_on_two_calls():
    import torch
    lib = tb.load_library()
    fn = lib.tm_window_stats_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p]
    n = 400000
    x = _waveform(n, 77)
    dx = torch.from_numpy(x).cuda()
    stream = torch.cuda.current_stream()
    with tb.Context(x) as ctx:
        for m in [1000, 72]:
            W = n - m + 1
            mean = torch.empty(W, dtype=torch.float32, device='cuda')
            std = torch.empty(W, dtype=torch.float32, device='cuda')
            flags = torch.empty(W, dtype=torch.uint8, device='cuda')
            rc = fn(dx.data_ptr(), n, m, mean.data_ptr(), std.data_ptr(), flags.data_ptr(), stream.cuda_stream)
            assert rc == 0
            torch.cuda.synchronize()
            ref_mean, ref_std = ctx.window_stats(m)
            got_mean, got_std, got_flags = mean.cpu().numpy(), std.cpu().numpy(), flags.cpu().numpy()
            missing = x[:W] == tb.MISSING_VALUE
            assert np.array_equal((got_flags & 1) != 0, missing)
            assert np.array_equal(got_std == 0, ref_std == 0)          # same constant / missing windows
            assert np.array_equal(((got_flags & 2) != 0), (ref_std == 0) & ~missing)
            scale = np.abs(ref_mean).astype(np.float64) + ref_std.astype(np.float64)
            assert np.all(np.abs(got_mean.astype(np.float64) - ref_mean) <= REL * scale)
            assert np.all(np.abs(got_std.astype(np.float64) - ref_std) <= REL * ref_std.astype(np.float64))
    too_big = torch.zeros(600000, dtype=torch.float32, device='cuda')
    out = torch.empty(600000, dtype=torch.float32, device='cuda')
    assert fn(too_big.data_ptr(), 600000, 100, out.data_ptr(), out.data_ptr(), out.data_ptr(), None) == -8
