// Length-independent window statistics: block-local FP64 prefix sums of the waveform and
// the length of the run of identical samples starting at every sample.
//
// The record is cut into blocks of kPrefixBlock samples, each with its own centre c_b (the
// block's mean, FP64). Within a block the sums restart:
//   Q[i] = (sum (x_t - c_b), sum (x_t - c_b)^2) over t from the start of i's block to i - 1,
// so Q[i] = 0 at every block start; T[b] holds block b's totals. A window [j, j + m) with
// m <= kPrefixBlock lies in one block or in two adjacent ones, so its sums come from at
// most one block total and two prefix values of those blocks (window_prefix_stats,
// tm_prefix.cuh). Their rounding errors are bounded by the magnitudes of those blocks
// alone: a loud stretch inflates the bounds of the windows near it, not of the rest of the
// record, and a block's centre follows a drifting offset.
//
// run[i] = number of consecutive samples equal to clean[i] starting at i (capped at
// 65535): a window is constant, hence not searchable (std 0 in the reference), exactly
// when run[j] >= m. Constant stretches (gaps filled with zeros, clipped data) are
// recognised without two-pass statistics.
#include "tm_prefix.cuh"

namespace tmb {

constexpr int PX_THREADS = 1024, PX_PER_THREAD = 8, PX_CHUNK = PX_THREADS * PX_PER_THREAD;
constexpr int PX_CHUNKS_PER_BLOCK = kPrefixBlock / PX_CHUNK;
static_assert(kPrefixBlock % PX_CHUNK == 0, "chunks tile the prefix blocks");

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

// The centred values of one thread's 8 samples (centres: one per prefix block, or null
// for 0) and their sum.
__device__ __forceinline__ double2 chunk_values(const float *__restrict__ clean, uint64_t n,
                                                const double *__restrict__ centres, uint64_t base, double2 *vals)
{
    const double c = centres ? centres[base >> kPrefixBlockLog] : 0.0; // 8 samples never straddle a block
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
__global__ void __launch_bounds__(PX_THREADS) k_prefix_totals(const float *__restrict__ clean, uint64_t n,
                                                              const double *__restrict__ centres,
                                                              double2 *__restrict__ totals)
{
    __shared__ double2 warp_tot[32];
    double2 vals[PX_PER_THREAD];
    const uint64_t base = (uint64_t)blockIdx.x * PX_CHUNK + (uint64_t)threadIdx.x * PX_PER_THREAD;
    const double2 s = block_scan(chunk_values(clean, n, centres, base, vals), warp_tot);
    if (threadIdx.x == blockDim.x - 1)
        totals[blockIdx.x] = s;
}

// Pass 2: within each prefix block, the exclusive scan of its chunks' totals (in place),
// and the block's totals T[b]. One thread per prefix block (8 chunks each).
__global__ void k_prefix_blocks(double2 *__restrict__ totals, uint32_t chunks, uint32_t blocks,
                                double2 *__restrict__ block_totals)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= blocks)
        return;
    double2 run = make_double2(0.0, 0.0);
    for (uint32_t c = b * PX_CHUNKS_PER_BLOCK; c < min(chunks, (b + 1) * PX_CHUNKS_PER_BLOCK); c++)
    {
        const double2 t = totals[c];
        totals[c] = run;
        run = add2(run, t);
    }
    block_totals[b] = run;
}

// Pass 3: Q[i + 1] for every sample (0 where i + 1 starts a block), Q[0] = 0.
__global__ void __launch_bounds__(PX_THREADS) k_prefix_apply(const float *__restrict__ clean, uint64_t n,
                                                             const double *__restrict__ centres,
                                                             const double2 *__restrict__ offsets,
                                                             double2 *__restrict__ Q)
{
    __shared__ double2 warp_tot[32];
    double2 vals[PX_PER_THREAD];
    const uint64_t base = (uint64_t)blockIdx.x * PX_CHUNK + (uint64_t)threadIdx.x * PX_PER_THREAD;
    const double2 s = chunk_values(clean, n, centres, base, vals);
    const double2 inc = block_scan(s, warp_tot);
    double2 run = add2(offsets[blockIdx.x], make_double2(inc.x - s.x, inc.y - s.y));
#pragma unroll
    for (int k = 0; k < PX_PER_THREAD; k++)
    {
        run = add2(run, vals[k]);
        const uint64_t i = base + k + 1;
        if (i <= n)
            Q[i] = (i & (kPrefixBlock - 1)) == 0 ? make_double2(0.0, 0.0) : run;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        Q[0] = make_double2(0.0, 0.0);
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

uint32_t prefix_chunks(uint64_t n) { return (uint32_t)((n + PX_CHUNK - 1) / PX_CHUNK); }

// Chunk totals (centres per prefix block, or null for 0); chunks = prefix_chunks(n).
cudaError_t launch_prefix_totals(const float *clean, uint64_t n, const double *centres, double2 *totals,
                                 cudaStream_t s)
{
    k_prefix_totals<<<prefix_chunks(n), PX_THREADS, 0, s>>>(clean, n, centres, totals);
    return cudaGetLastError();
}

// Q (n + 1 entries) and T (blocks entries) with the given centres; totals: scratch of
// prefix_chunks(n) entries.
cudaError_t launch_prefix_sums(const float *clean, uint64_t n, const double *centres, double2 *totals,
                               double2 *block_totals, double2 *Q, cudaStream_t s)
{
    const uint32_t chunks = prefix_chunks(n);
    const uint32_t blocks = (uint32_t)((n + kPrefixBlock - 1) / kPrefixBlock);
    k_prefix_totals<<<chunks, PX_THREADS, 0, s>>>(clean, n, centres, totals);
    k_prefix_blocks<<<(blocks + 255) / 256, 256, 0, s>>>(totals, chunks, blocks, block_totals);
    k_prefix_apply<<<chunks, PX_THREADS, 0, s>>>(clean, n, centres, totals, Q);
    return cudaGetLastError();
}

// run and run_tmp: n uint16 each; the result ends in `run`.
cudaError_t launch_runs(const float *clean, uint64_t n, uint16_t *run, uint16_t *run_tmp, cudaStream_t s)
{
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
