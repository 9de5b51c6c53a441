// Window statistics for one template length m.
//
// The reference computes, per window, an exact two-pass FP64 mean and population
// std and keeps them as float (SkipSequential.cpp:157-190; indexing.cpp:128-152;
// DMASS_V3.c:854-873), because global prefix sums lose every significant digit in
// quiet windows that follow loud samples (indexing.cpp:130-132).
//
// Here the sums come from FP64 *segmented* prefix sums with segments of exactly m
// samples: a window starting at offset o of segment a covers the suffix of segment
// a from o and the prefix of segment a+1 up to o-1, so
//     sum(window) = SUF_a[o] + PRE_{a+1}[o-1]
// and both terms accumulate only the window's own samples: no subtraction of large
// running sums, no cancellation from loud samples elsewhere. The one-pass variance
// E[x^2] - mean^2 can still cancel when |mean| >> std; such windows, and windows whose
// std is near the reference's 1e-12 degeneracy cut, are flagged and recomputed with
// the reference's own two-pass arithmetic (k_exact_stats), which also makes the
// degeneracy decision bit-identical to the reference.
#include "tm_internal.cuh"
#include "tm_exact.cuh"

namespace tmb {

__global__ void k_clean(const float *__restrict__ raw, float *__restrict__ clean, uint64_t n, uint64_t n_total)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_total;
         i += (uint64_t)gridDim.x * blockDim.x)
    {
        float v = i < n ? raw[i] : 0.0f;
        clean[i] = v == kMissing ? 0.0f : v;
    }
}

// One warp per segment [a*m, (a+1)*m) ∩ [0, n): suffix sums of (x, x^2) in FP64.
// suf is indexed relative to sbase = a_lo * m.
__global__ void k_segment_suffix(const float *__restrict__ clean, uint64_t n, int m, uint64_t a_lo, uint64_t a_count,
                                 double2 *__restrict__ suf)
{
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= a_count)
        return;
    const uint64_t a = a_lo + warp;
    const uint64_t base = a * (uint64_t)m;
    const uint64_t end = min(base + (uint64_t)m, n); // exclusive
    const uint64_t sbase = a_lo * (uint64_t)m;
    double cs = 0.0, cq = 0.0; // carry: sums of the part right of the current chunk
    for (int64_t hi = (int64_t)end; hi > (int64_t)base; hi -= 32)
    {
        const int64_t idx = hi - 32 + lane;
        const bool valid = idx >= (int64_t)base;
        const double v = valid ? (double)clean[idx] : 0.0;
        double s = v, q = v * v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const double ts = __shfl_down_sync(0xffffffffu, s, off);
            const double tq = __shfl_down_sync(0xffffffffu, q, off);
            if (lane + off < 32)
            {
                s += ts;
                q += tq;
            }
        }
        if (valid)
            suf[idx - (int64_t)sbase] = make_double2(s + cs, q + cq);
        cs += __shfl_sync(0xffffffffu, s, 0);
        cq += __shfl_sync(0xffffffffu, q, 0);
    }
}

__device__ __forceinline__ void finalize_window(uint64_t j, uint64_t w0, int m, double s, double q,
                                                const float *__restrict__ raw, float *__restrict__ mean,
                                                float *__restrict__ inv, uint8_t *__restrict__ flags, double r2max)
{
    const uint64_t r = j - w0;
    if (raw[j] == kMissing)
    {
        mean[r] = 0.0f;
        inv[r] = 0.0f;
        flags[r] = kFlagMissingStart;
        return;
    }
    const double mu = s / (double)m;
    const double var = q / (double)m - mu * mu;
    // relative error of var is about m * eps64 * (1 + 2 mu^2 / var); trust it up to ~1e-6
    const bool cancel = !(var > 0.0) || mu * mu > var * r2max;
    const bool tiny = var < 1e-22; // std < 1e-11: decide degeneracy (<= 1e-12) exactly
    if (cancel || tiny)
    {
        mean[r] = (float)mu;
        inv[r] = 0.0f;
        flags[r] = kFlagNeedsExact;
        return;
    }
    mean[r] = (float)mu;
    inv[r] = (float)(1.0 / sqrt(var));
    flags[r] = 0;
}

// One warp per segment a: windows j = a*m + o, o in [0, m), restricted to [w0, w0 + W).
__global__ void k_window_stats(const float *__restrict__ clean, const float *__restrict__ raw,
                               const double2 *__restrict__ suf, uint64_t n, int m, uint64_t a_lo, uint64_t a_count,
                               uint64_t w0, uint64_t W, float *__restrict__ mean, float *__restrict__ inv,
                               uint8_t *__restrict__ flags, double r2max)
{
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= a_count)
        return;
    const uint64_t a = a_lo + warp;
    const uint64_t base = a * (uint64_t)m;
    const uint64_t sbase = a_lo * (uint64_t)m;
    const uint64_t wend = w0 + W;
    if (lane == 0 && base >= w0 && base < wend)
    {
        const double2 v = suf[base - sbase];
        finalize_window(base, w0, m, v.x, v.y, raw, mean, inv, flags, r2max);
    }
    double cs = 0.0, cq = 0.0; // carry: prefix of segment a+1
    for (int p0 = 0; p0 < m - 1; p0 += 32)
    {
        const int p = p0 + lane;
        const uint64_t j = base + (uint64_t)p + 1;      // window start
        const uint64_t idx = base + (uint64_t)m + p;    // = j + m - 1, last sample of window j
        const bool in_seg = p < m - 1 && idx < n;
        const double v = in_seg ? (double)clean[idx] : 0.0;
        double s = v, q = v * v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const double ts = __shfl_up_sync(0xffffffffu, s, off);
            const double tq = __shfl_up_sync(0xffffffffu, q, off);
            if (lane >= off)
            {
                s += ts;
                q += tq;
            }
        }
        s += cs;
        q += cq;
        if (in_seg && j >= w0 && j < wend)
        {
            const double2 sv = suf[j - sbase];
            finalize_window(j, w0, m, sv.x + s, sv.y + q, raw, mean, inv, flags, r2max);
        }
        cs = __shfl_sync(0xffffffffu, s, 31);
        cq = __shfl_sync(0xffffffffu, q, 31);
        if (base + (uint64_t)p0 + 33 >= wend)
            break; // every later window of this segment is past the range
    }
}

// Fix-up of flagged windows with the reference's exact statistics.
__global__ void k_exact_stats(const float *__restrict__ raw, int m, uint64_t w0, uint64_t W, float *__restrict__ mean,
                              float *__restrict__ inv, uint8_t *__restrict__ flags)
{
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < W; r += (uint64_t)gridDim.x * blockDim.x)
    {
        if (!(flags[r] & kFlagNeedsExact))
            continue;
        float mf, sf;
        exact_stats(raw, w0 + r, m, mf, sf);
        mean[r] = mf;
        if (sf == 0.0f)
        {
            inv[r] = 0.0f;
            flags[r] = kFlagDegenerate | kFlagExact;
        }
        else
        {
            inv[r] = (float)(1.0 / (double)sf);
            flags[r] = kFlagExact;
        }
    }
}

// Exact float statistics of windows [w0, w0 + count) (the reference's stored values).
__global__ void k_reference_stats(const float *__restrict__ raw, int m, uint64_t w0, uint64_t count,
                                  float *__restrict__ mean, float *__restrict__ stddev)
{
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < count;
         r += (uint64_t)gridDim.x * blockDim.x)
    {
        if (raw[w0 + r] == kMissing)
        {
            mean[r] = 0.0f;
            stddev[r] = 0.0f;
            continue;
        }
        float mf, sf;
        exact_stats(raw, w0 + r, m, mf, sf);
        mean[r] = mf;
        stddev[r] = sf;
    }
}

// ---- launchers --------------------------------------------------------------------

cudaError_t launch_clean(const float *raw, float *clean, uint64_t n, uint64_t n_total, cudaStream_t s)
{
    k_clean<<<1184, 256, 0, s>>>(raw, clean, n, n_total);
    return cudaGetLastError();
}

// suf must hold (a_count * m) double2.
cudaError_t launch_window_stats(const float *clean, const float *raw, uint64_t n, int m, uint64_t w0, uint64_t W,
                                double2 *suf, float *mean, float *inv, uint8_t *flags, cudaStream_t s)
{
    const uint64_t a_lo = w0 / (uint64_t)m;
    const uint64_t a_hi = (w0 + W - 1) / (uint64_t)m;
    const uint64_t a_count = a_hi - a_lo + 1;
    const int threads = 256;
    const uint64_t blocks = (a_count * 32 + threads - 1) / threads;
    k_segment_suffix<<<(unsigned)blocks, threads, 0, s>>>(clean, n, m, a_lo, a_count, suf);
    const double r2max = 5e-7 / ((double)m * 1.1102230246251565e-16);
    k_window_stats<<<(unsigned)blocks, threads, 0, s>>>(clean, raw, suf, n, m, a_lo, a_count, w0, W, mean, inv, flags,
                                                        r2max);
    k_exact_stats<<<1184, 256, 0, s>>>(raw, m, w0, W, mean, inv, flags);
    return cudaGetLastError();
}

cudaError_t launch_reference_stats(const float *raw, int m, uint64_t w0, uint64_t count, float *mean, float *stddev,
                                   cudaStream_t s)
{
    k_reference_stats<<<1184, 128, 0, s>>>(raw, m, w0, count, mean, stddev);
    return cudaGetLastError();
}

} // namespace tmb
