// Length-independent window statistics: FP64 prefix sums of the waveform and the
// length of the run of identical samples starting at every sample.
//
// P[i] = (sum_{t<i} (x_t - c), sum_{t<i} (x_t - c)^2), i = 0..n, with c the mean of the
// clean waveform (missing samples are 0) so that an offset does not inflate the sums.
// A window [j, j+m) then has s1 = P1[j+m] - P1[j] and s2 = P2[j+m] - P2[j] for any m,
// which is what lets templates of different lengths share one contraction tile. The
// subtraction can cancel (a quiet window after loud samples); every use bounds that
// error (window_stats_from_prefix in tm_prefix.cuh) and hands doubtful windows to the
// exact re-scoring.
//
// run[i] = number of consecutive samples equal to clean[i] starting at i (capped at
// 65535): a window is constant, hence not searchable (std 0 in the reference), exactly
// when run[j] >= m. Constant stretches (gaps filled with zeros, clipped data) are
// recognised without two-pass statistics.
#include "tm_internal.cuh"

namespace tmb {

constexpr int PX_THREADS = 1024, PX_PER_THREAD = 8, PX_CHUNK = PX_THREADS * PX_PER_THREAD;

__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// Block-wide inclusive scan of one double2 per thread.
__device__ double2 block_scan(double2 v, double2 *warp_tot)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        const double a = __shfl_up_sync(0xffffffffu, v.x, off), b = __shfl_up_sync(0xffffffffu, v.y, off);
        if (lane >= off)
            v = add2(v, make_double2(a, b));
    }
    if (lane == 31)
        warp_tot[warp] = v;
    __syncthreads();
    if (warp == 0)
    {
        double2 w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : make_double2(0.0, 0.0);
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const double a = __shfl_up_sync(0xffffffffu, w.x, off), b = __shfl_up_sync(0xffffffffu, w.y, off);
            if (lane >= off)
                w = add2(w, make_double2(a, b));
        }
        warp_tot[lane] = w; // inclusive warp totals
    }
    __syncthreads();
    if (warp > 0)
        v = add2(v, warp_tot[warp - 1]);
    return v;
}

__device__ __forceinline__ double2 chunk_values(const float *__restrict__ clean, uint64_t n, double c, uint64_t base,
                                                double2 *vals)
{
    double2 s = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < PX_PER_THREAD; k++)
    {
        const uint64_t i = base + k;
        const double v = i < n ? (double)clean[i] - c : 0.0;
        vals[k] = make_double2(v, i < n ? v * v : 0.0);
        s = add2(s, vals[k]);
    }
    return s;
}

// Pass 1: per-chunk totals.
__global__ void __launch_bounds__(PX_THREADS) k_prefix_totals(const float *__restrict__ clean, uint64_t n, double c,
                                                              double2 *__restrict__ totals)
{
    __shared__ double2 warp_tot[32];
    double2 vals[PX_PER_THREAD];
    const uint64_t base = (uint64_t)blockIdx.x * PX_CHUNK + (uint64_t)threadIdx.x * PX_PER_THREAD;
    const double2 s = block_scan(chunk_values(clean, n, c, base, vals), warp_tot);
    if (threadIdx.x == blockDim.x - 1)
        totals[blockIdx.x] = s;
}

// Pass 2 (one block): exclusive scan of the chunk totals, in place.
__global__ void __launch_bounds__(PX_THREADS) k_prefix_scan_totals(double2 *__restrict__ totals, uint32_t chunks)
{
    __shared__ double2 warp_tot[32];
    __shared__ double2 carry;
    if (threadIdx.x == 0)
        carry = make_double2(0.0, 0.0);
    __syncthreads();
    for (uint32_t b = 0; b < chunks; b += PX_THREADS)
    {
        const uint32_t i = b + threadIdx.x;
        const double2 v = i < chunks ? totals[i] : make_double2(0.0, 0.0);
        const double2 inc = block_scan(v, warp_tot);
        const double2 c0 = carry;
        if (i < chunks)
            totals[i] = add2(c0, make_double2(inc.x - v.x, inc.y - v.y));
        __syncthreads();
        if (threadIdx.x == PX_THREADS - 1)
            carry = add2(c0, inc);
        __syncthreads();
    }
}

// Pass 3: P[i + 1] for every sample, P[0] = 0.
__global__ void __launch_bounds__(PX_THREADS) k_prefix_apply(const float *__restrict__ clean, uint64_t n, double c,
                                                             const double2 *__restrict__ offsets,
                                                             double2 *__restrict__ P)
{
    __shared__ double2 warp_tot[32];
    double2 vals[PX_PER_THREAD];
    const uint64_t base = (uint64_t)blockIdx.x * PX_CHUNK + (uint64_t)threadIdx.x * PX_PER_THREAD;
    const double2 s = chunk_values(clean, n, c, base, vals);
    const double2 inc = block_scan(s, warp_tot);
    double2 run = add2(offsets[blockIdx.x], make_double2(inc.x - s.x, inc.y - s.y));
#pragma unroll
    for (int k = 0; k < PX_PER_THREAD; k++)
    {
        run = add2(run, vals[k]);
        if (base + k < n)
            P[base + k + 1] = run;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        P[0] = make_double2(0.0, 0.0);
}

// run[i]: samples equal to clean[i] from i on, capped. Round 0 looks ahead up to 16
// samples; each later round doubles the cap by pointer jumping: a run that reaches the
// cap continues with the (capped) run of the sample cap positions later when that sample
// has the same value. O(n log cap) in every case, constant stretches included.
__global__ void k_run_init(const float *__restrict__ clean, uint64_t n, uint16_t *__restrict__ run)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    {
        const float v = clean[i];
        uint32_t len = 1;
        while (len < 16u && i + len < n && clean[i + len] == v)
            len++;
        run[i] = (uint16_t)len;
    }
}

__global__ void k_run_double(const float *__restrict__ clean, uint64_t n, uint32_t cap,
                             const uint16_t *__restrict__ in, uint16_t *__restrict__ out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    {
        uint32_t len = in[i];
        if (len == cap && i + cap < n && clean[i + cap] == clean[i])
            len += in[i + cap];
        out[i] = (uint16_t)min(len, 65535u);
    }
}

// totals: ceil(n / 8192) double2; P: n + 1 double2; run and run_tmp: n uint16 each.
cudaError_t launch_prefix(const float *clean, uint64_t n, double c, double2 *totals, double2 *P, uint16_t *run,
                          uint16_t *run_tmp, cudaStream_t s)
{
    const uint32_t chunks = (uint32_t)((n + PX_CHUNK - 1) / PX_CHUNK);
    k_prefix_totals<<<chunks, PX_THREADS, 0, s>>>(clean, n, c, totals);
    k_prefix_scan_totals<<<1, PX_THREADS, 0, s>>>(totals, chunks);
    k_prefix_apply<<<chunks, PX_THREADS, 0, s>>>(clean, n, c, totals, P);
    // 16 -> 32 -> ... -> 65536: 12 doublings, an even number, so the result ends in `run`
    k_run_init<<<1184, 256, 0, s>>>(clean, n, run);
    uint16_t *a = run, *b = run_tmp;
    for (uint32_t cap = 16; cap < 65536u; cap *= 2)
    {
        k_run_double<<<1184, 256, 0, s>>>(clean, n, cap, a, b);
        uint16_t *t = a;
        a = b;
        b = t;
    }
    return cudaGetLastError();
}

} // namespace tmb
