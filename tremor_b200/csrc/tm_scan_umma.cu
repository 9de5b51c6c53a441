// Split-BF16 tensor-core contraction (tcgen05, sm_100a) with the fused bounded epilogue.
//
// Work: D[t][j] = sum_i q_t[i] (x_{j+i} - s) for 128 templates (M, TMEM lanes) x 256
// windows (N, TMEM columns) per tile, over K = m. FP32 products are recovered from
// BF16 halves: q = q_hi + q_lo, (x - s) = x_hi + x_lo, and
//     q (x - s) ~= q_hi x_hi + q_hi x_lo + q_lo x_hi       (3 MMAs per K step)
// with products exact in the tensor core and FP32 accumulation in TMEM; the dropped
// and rounding terms are below 3.01 * 2^-18 |q||x - s| per product and enter the
// per-result error bound (gamma_bf16 on the host).
//
// Operands in shared memory:
//   A (templates, K-major): TMA tiles of 128 rows x 64 samples, SWIZZLE_128B, hi and lo.
//   B (windows, K-major): the Hankel matrix H[j][k] = x[j0 + k0 + j + k]. In the
//     canonical no-swizzle K-major layout a core matrix is 8 rows x 16 bytes, rows 16
//     bytes apart; core matrix (row group g, K chunk c) of H holds x[8(g+c) + r + e]
//     and so depends on g + c only. One strip of core matrices
//         U[u][r][e] = x[k0 + 8u + r + e],   u = 0 .. N/8 + 64/8 - 1,
//     described with SBO (between row groups) = LBO (between K chunks) = 128 bytes,
//     is the whole 256 x 64 Hankel tile: the descriptor's overlapping core matrices
//     supply the one-sample shift from row to row that no byte stride can express.
//     Builder warps write the strip (hi and lo) from the waveform each stage.
//
// Warp roles (384 threads): warp 0 TMA producer, warp 1 TMEM owner + MMA issuer,
// warps 2-3 strip builders, warps 4-11 epilogue (TMEM lane quarter = warp % 4; warps w and
// w + 4 split the tile's 256 columns).
// Pipelines: S smem stages (full_a / full_b / empty mbarriers), two TMEM accumulators
// of 256 columns (acc_full / acc_empty), persistent CTAs over (template tile, window
// tile) pairs, template-tile-major so a tile's templates stay in L2.
//
// Every wait is bounded: after about a second without progress the CTA records an
// error in *err, every role leaves its loop, and TMEM is released before exit.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "tm_epilogue.cuh"
#include "tm_prefix.cuh"

namespace tmb {

namespace umma {

constexpr int TM = 128;       // templates per tile (MMA M)
constexpr int TN = 256;       // windows per tile (MMA N)
constexpr int KB = 64;        // samples per stage (one 128-byte swizzle atom of BF16)
constexpr int STRIP_CHUNKS = TN / 8 + KB / 8; // 40 core matrices of 128 bytes
constexpr int A_BYTES = TM * KB * 2;          // 16 KiB per half
constexpr int B_BYTES = STRIP_CHUNKS * 128;   // 5 KiB per half
constexpr int THREADS = 384;  // 4 role warps + 8 epilogue warps
constexpr int BUILDERS = 64;
constexpr int EPI = 256;      // epilogue threads
constexpr uint32_t TMEM_COLS = 2 * TN;
constexpr long long TIMEOUT_CYCLES = 4000000000ll; // ~2 s at 2 GHz

// Shared memory. Single-length tiles stage the per-window statistics of their length
// (double-buffered by tile). Mixed-length tiles keep, per epilogue warp, the distinct
// lengths of its 32 template rows and the statistics of its current group of windows for
// each of those lengths; no other role reads them.
template <bool MIXED> struct SmemT
{
    static constexpr int S = 4;                 // operand stages
    static constexpr int W2 = MIXED ? 1 : 2;    // single-length window statistics buffers
    static constexpr int WL = MIXED ? 8 : 1;    // mixed: per-warp tables
    static constexpr uint32_t STAGE = MIXED ? 128 : 256; // staged candidates per epilogue warp
    uint8_t a_hi[S][A_BYTES]; // 1024-byte aligned (swizzle atoms)
    uint8_t a_lo[S][A_BYTES];
    uint8_t b_hi[S][B_BYTES];
    uint8_t b_lo[S][B_BYTES];
    // window terms (1/sigma, mu - shift, E0, 0) of window i of a group of G windows for
    // distinct length d at [warp][d G + (i ^ (d & 7))] (G x d <= 256): lanes reading
    // different lengths for the same window hit different banks
    float4 wst[WL][256];
    int wl_len[WL][32];        // the warp's distinct lengths
    uint32_t wl_wc[WL][32];    //   their window counts in the searched range
    double wl_inv[WL][32];     //   their inverses
    float wl_fim[WL][32];      //   the same in float, rounded up
    float4 wl_c[WL][32];       //   maxima over their rows of a1, a5, a6 and 1.25 (4 m + 2 qs)
    float wl_b[WL][32];        //   and of 2.5 |s1|
    float4 win4[W2][TN];       // single-length tiles: window terms (win_terms), then (1/sigma, mu - shift, eb, Q)
    float win_h[W2][TN];
    float4 coef[8];            // single-length tiles: per epilogue warp, maxima over its rows of (a1, a45, a6, c24)
    Candidate stage[8][STAGE]; // per epilogue warp: candidates before their flush
    uint64_t full_a[S], full_b[S], empty[S];
    uint64_t acc_full[2], acc_empty[2], win_ready[2], eb_ready[2], drain;
    uint32_t tmem_base;
    int abort;
};

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(saddr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// try_wait with a suspend-time hint (ns): a waiting warp sleeps until the phase completes
// or the hint runs out, instead of re-polling and taking issue slots from the warps it
// waits for.
__device__ __forceinline__ bool mbar_try_sleep(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(saddr(bar)), "r"(parity), "r"(20000u)
                 : "memory");
    return ok != 0;
}
// Bounded wait: false on timeout or when another role aborted (the CTA then unwinds).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int &abort_flag, int *err, int where)
{
    if (mbar_try(bar, parity))
        return true;
    const long long t0 = clock64();
    while (true)
    {
        if (mbar_try_sleep(bar, parity))
            return true;
        if (*(volatile int *)&abort_flag)
            return false;
        if (clock64() - t0 > TIMEOUT_CYCLES)
        {
            *(volatile int *)&abort_flag = 1;
            atomicExch(err, 1000 + where);
            return false;
        }
    }
}

// mbar_wait agreed by the whole warp: every lane continues only if all lanes succeeded, so a
// warp-collective instruction after the wait is never reached by part of a warp.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity, int &abort_flag, int *err, int where)
{
    return __all_sync(0xffffffffu, mbar_wait(bar, parity, abort_flag, err, where));
}

// Short bounded wait used while unwinding after an abort (ignores the abort flag).
__device__ __forceinline__ void mbar_drain(uint64_t *bar, uint32_t parity)
{
    const long long t0 = clock64();
    while (!mbar_try(bar, parity) && clock64() - t0 < TIMEOUT_CYCLES / 8)
        ;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                 "[%4];" ::"r"(saddr(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr(bar))
                 : "memory");
}

// Shared-memory matrix descriptor (tcgen05): start, LBO, SBO in 16-byte units,
// version 1, layout type in bits 61-63 (0: no swizzle, 2: 128-byte swizzle).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major, N = 256, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
                 "l"(a), "l"(b), "r"(IDESC), "r"(accumulate)
                 : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                 "%14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++)
        v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v)
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; i++)
        v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b); // .x = a (low half), .y = b
    return *reinterpret_cast<const uint32_t *>(&h);
}

static_assert(sizeof(SmemT<false>) + 1024 <= 227 * 1024, "shared memory of k_scan_umma");
static_assert(sizeof(SmemT<true>) + 1024 <= 227 * 1024, "shared memory of k_scan_umma (mixed)");

struct UmmaArgs
{
    ScanArgs a;
    int t_tiles, w_tiles, kblocks;
    int *err;
};

// Tile shift (the value subtracted from the waveform before the split): the mean of the
// middle window for single-length launches; for mixed-length tiles the middle sample.
template <bool MIXED> __device__ __forceinline__ float tile_shift(const ScanArgs &a, uint32_t j0)
{
    const uint32_t jm = min(j0 + TN / 2, a.W - 1);
    return MIXED ? a.x[a.w0 + jm] : a.mean[jm];
}

// The bound of fast_distance (tm_epilogue.cuh) with its window-only factors hoisted out
// of the per-pair loop:
//   e = a1 S + a2 + a3 max(d, 0) + a4 (1 + 2 Q) + a5 Q + a6 H,
//   S = sqrt(1 + r^2), r = (mu - shift) / sigma, Q = (mu / sigma)^2, H = (|mu| + |shift|) / sigma,
// evaluated as e = a3 max(d, 0) + eb with eb = a1 S + (2 a4 + a5) Q + a6 H + (a2 + a4).
// Window terms: (1/sigma, mu - shift, S, Q) and H. A window that is not searched has
// 1/sigma = 0 and S = NaN: its e, d - e and d + e are NaN, which no threshold comparison
// accepts and fminf ignores, so the per-pair code needs no branch.
__device__ __forceinline__ float nan_f() { return __int_as_float(0x7fc00000); }

__device__ __forceinline__ float4 skip_terms(float &h)
{
    h = 0.0f;
    return make_float4(0.0f, 0.0f, nan_f(), 0.0f);
}

__device__ __forceinline__ float4 win_terms(float mu, float iv, float shift, float &h)
{
    if (iv == 0.0f)
        return skip_terms(h);
    const float ms = mu - shift;
    const float r = ms * iv, r0 = mu * iv;
    h = (fabsf(mu) + fabsf(shift)) * iv;
    return make_float4(iv, ms, sqrtf(1.0f + r * r), r0 * r0);
}

// Per-template (lane) constants of the hoisted bound. thr is the threshold on d - e, NaN
// for kNN templates and padding rows (no window passes it).
struct LaneTerms
{
    float s1, c_lin, a1, a3, a45, a6, c24, a2, thr;
};

__device__ __forceinline__ LaneTerms lane_terms(const TemplParam &p, bool valid)
{
    LaneTerms l;
    l.s1 = p.s1;
    l.c_lin = p.c_lin;
    l.a1 = p.a1_main;
    l.a3 = p.a3;
    l.a45 = 2.0f * p.a4 + p.a5;
    l.a6 = p.a6;
    l.c24 = p.a2 + p.a4;
    l.a2 = p.a2;
    l.thr = (valid && p.mode != 1) ? p.thr_ed : nan_f();
    return l;
}

// Mixed-length tiles: the window terms of one (window, length) from its statistics and
// the length's coefficient maxima c = (a1, a5, a6, 1.25 (4 m + 2 qs)) and cb = 2.5 |s1|:
// (1/sigma, mu - shift, E0, 0) with E0 = the window part of fast_distance_mixed's bound
// without a2 (a1 S + a5 Q + a6 H + the statistics' own error term of stats_error). With
// the maxima over the length's rows in place of each row's own coefficients, E0 bounds
// that part for every row of the length.
__device__ __forceinline__ float4 mixed_terms(const WindowStats &ws, float shift, float4 c, float cb)
{
    const float ms = ws.mu - shift;
    const float r = ms * ws.iv, r0 = ws.mu * ws.iv;
    const float e0 = c.x * sqrtf(1.0f + r * r) + c.y * (r0 * r0) + c.z * (fabsf(ws.mu) + fabsf(shift)) * ws.iv +
                     c.w * ws.rel_sd + cb * (ws.e_mu * ws.iv);
    return make_float4(ws.iv, ms, e0, 0.0f);
}

// mixed_terms for statistics from the fast path (prefix_stats_fast): the relative error of
// the std is at most kFastRelSd, and sqrt(1 + r^2) <= 1 + |r|.
__device__ __forceinline__ float4 mixed_terms_fast(float mu, float iv, float e_mu, float shift, float4 c, float cb)
{
    const float ms = mu - shift;
    const float r = ms * iv, r0 = mu * iv;
    const float e0 = c.x * (1.0f + fabsf(r)) + c.y * (r0 * r0) + c.z * (fabsf(mu) + fabsf(shift)) * iv +
                     c.w * kFastRelSd + cb * (e_mu * iv);
    return make_float4(iv, ms, e0, 0.0f);
}

// Maximum of a non-negative float over the lanes where `mine` holds (0 when none).
__device__ __forceinline__ float warp_max_nonneg(bool mine, float v)
{
    return __uint_as_float(__reduce_max_sync(0xffffffffu, mine ? __float_as_uint(v) : 0u));
}

// d and e of one pair from its shifted dot product (fast_distance's d, evaluated the same
// way) and the window part eb of its bound.
__device__ __forceinline__ void pair_bound(const LaneTerms &l, float dot, float iv, float ms, float eb, float &d,
                                           float &e)
{
    const float cross = (dot - ms * l.s1) * iv;
    d = l.c_lin - 2.0f * cross;
    e = fmaf(l.a3, fmaxf(d, 0.0f), eb);
}

// Threshold bit i of mask when d - e <= thr; kNN bucket minima of d + e and d - e (used
// only for kNN rows).
__device__ __forceinline__ void pair_update(const LaneTerms &l, float dot, float iv, float ms, float eb, int i,
                                            uint32_t &mask, float &umin, float &lmin)
{
    float d, e;
    pair_bound(l, dot, iv, ms, eb, d, e);
    const float lo = d - e;
    umin = fminf(umin, d + e);
    lmin = fminf(lmin, lo);
    mask |= (lo <= l.thr ? 1u : 0u) << i;
}

template <bool MIXED>
__global__ void __launch_bounds__(THREADS, 1)
    k_scan_umma(const UmmaArgs ua, const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    using Sm = SmemT<MIXED>;
    constexpr int STAGES = Sm::S;
    Sm &sm = *reinterpret_cast<Sm *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const ScanArgs &a = ua.a;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long tiles = (long long)ua.t_tiles * ua.w_tiles;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < STAGES; s++)
        {
            mbar_init(&sm.full_a[s], 1);
            mbar_init(&sm.full_b[s], BUILDERS);
            mbar_init(&sm.empty[s], 1);
        }
        for (int b = 0; b < 2; b++)
        {
            mbar_init(&sm.acc_full[b], 1);
            mbar_init(&sm.acc_empty[b], EPI);
            mbar_init(&sm.win_ready[b], EPI);
            mbar_init(&sm.eb_ready[b], EPI);
        }
        mbar_init(&sm.drain, 1);
        sm.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&sm.tmem_base)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;

    if (warp == 0)
    {
        // ---- TMA producer: template tiles (hi, lo) ----
        if (lane == 0)
        {
            uint32_t it = 0;
            for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x)
            {
                const int tt = (int)(tile / ua.w_tiles);
                const int kblocks = MIXED ? a.tiles[tt].kb : ua.kblocks;
                for (int kb = 0; kb < kblocks; kb++, it++)
                {
                    const int s = it % STAGES;
                    if (!mbar_wait(&sm.empty[s], ((it / STAGES) & 1) ^ 1, sm.abort, ua.err, 1))
                    {
                        // unwinding: let the copies already issued land before the CTA exits
                        for (uint32_t i = it > STAGES ? it - STAGES : 0; i < it; i++)
                            mbar_drain(&sm.full_a[i % STAGES], (i / STAGES) & 1);
                        goto done;
                    }
                    mbar_expect_tx(&sm.full_a[s], 2 * A_BYTES);
                    tma_load_2d(sm.a_hi[s], &map_hi, kb * KB, tt * TM, &sm.full_a[s]);
                    tma_load_2d(sm.a_lo[s], &map_lo, kb * KB, tt * TM, &sm.full_a[s]);
                }
            }
        }
    }
    else if (warp == 1)
    {
        // ---- MMA issuer ----
        if (lane == 0)
        {
            uint32_t it = 0, tc = 0;
            for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x, tc++)
            {
                const int buf = tc & 1;
                if (!mbar_wait(&sm.acc_empty[buf], ((tc >> 1) & 1) ^ 1, sm.abort, ua.err, 2))
                {
                    mma_commit(&sm.drain);
                    mbar_drain(&sm.drain, 0);
                    goto done;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(buf * TN);
                const int kblocks = MIXED ? a.tiles[tile / ua.w_tiles].kb : ua.kblocks;
                for (int kb = 0; kb < kblocks; kb++, it++)
                {
                    const int s = it % STAGES;
                    const uint32_t ph = (it / STAGES) & 1;
                    if (!mbar_wait(&sm.full_a[s], ph, sm.abort, ua.err, 3) || !mbar_wait(&sm.full_b[s], ph, sm.abort, ua.err, 4))
                    {
                        // unwinding: wait for the MMAs already issued before TMEM is released
                        mma_commit(&sm.drain);
                        mbar_drain(&sm.drain, 0);
                        goto done;
                    }
                    tc_fence_after();
                    const uint32_t ah = saddr(sm.a_hi[s]), al = saddr(sm.a_lo[s]);
                    const uint32_t bh = saddr(sm.b_hi[s]), bl = saddr(sm.b_lo[s]);
#pragma unroll
                    for (int kk = 0; kk < KB / 16; kk++)
                    {
                        const uint64_t dah = sdesc(ah + kk * 32, 16, 1024, 2);
                        const uint64_t dal = sdesc(al + kk * 32, 16, 1024, 2);
                        const uint64_t dbh = sdesc(bh + kk * 256, 128, 128, 0);
                        const uint64_t dbl = sdesc(bl + kk * 256, 128, 128, 0);
                        mma(d, dah, dbh, (kb | kk) != 0);
                        mma(d, dah, dbl, 1);
                        mma(d, dal, dbh, 1);
                    }
                    mma_commit(&sm.empty[s]); // frees the stage when these MMAs complete
                }
                mma_commit(&sm.acc_full[buf]);
            }
        }
    }
    else if (warp < 4)
    {
        // ---- strip builders: U[u][r][e] = split(x[base + 8u + r + e] - shift) ----
        const int tid = threadIdx.x - 64;
        uint32_t it = 0;
        for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x)
        {
            const uint32_t j0 = (uint32_t)(tile % ua.w_tiles) * TN;
            const float shift = tile_shift<MIXED>(a, j0);
            const float *xw = a.x + a.w0 + j0;
            const int kblocks = MIXED ? a.tiles[tile / ua.w_tiles].kb : ua.kblocks;
            for (int kb = 0; kb < kblocks; kb++, it++)
            {
                const int s = it % STAGES;
                if (!mbar_wait(&sm.empty[s], ((it / STAGES) & 1) ^ 1, sm.abort, ua.err, 5))
                    goto done;
                const float *xs = xw + kb * KB;
                for (int row = tid; row < STRIP_CHUNKS * 8; row += BUILDERS)
                {
                    const int u = row >> 3, r = row & 7;
                    float v[8], h[8], l[8];
#pragma unroll
                    for (int e = 0; e < 8; e++)
                        v[e] = xs[8 * u + r + e] - shift;
#pragma unroll
                    for (int e = 0; e < 8; e++)
                    {
                        h[e] = __bfloat162float(__float2bfloat16_rn(v[e]));
                        l[e] = v[e] - h[e];
                    }
                    uint4 hv, lv;
                    hv.x = pack_bf16(h[0], h[1]);
                    hv.y = pack_bf16(h[2], h[3]);
                    hv.z = pack_bf16(h[4], h[5]);
                    hv.w = pack_bf16(h[6], h[7]);
                    lv.x = pack_bf16(l[0], l[1]);
                    lv.y = pack_bf16(l[2], l[3]);
                    lv.z = pack_bf16(l[4], l[5]);
                    lv.w = pack_bf16(l[6], l[7]);
                    *reinterpret_cast<uint4 *>(&sm.b_hi[s][u * 128 + r * 16]) = hv;
                    *reinterpret_cast<uint4 *>(&sm.b_lo[s][u * 128 + r * 16]) = lv;
                }
                fence_proxy_async(); // generic-proxy smem writes -> visible to the tensor core
                mbar_arrive(&sm.full_b[s]);
            }
        }
    }
    else
    {
        // ---- epilogue (8 warps): TMEM -> distances, bounds, candidates / bucket minima ----
        // Warps w and w + 4 read the same TMEM lane quarter (warp % 4) and split the columns.
        const int quarter = warp & 3;
        const int ew = warp - 4;              // epilogue warp 0..7
        const int half = ew >> 2;
        const int row = quarter * 32 + lane;  // TMEM lane = template row within the tile
        const int et = threadIdx.x - 128;     // 0..255
        constexpr uint32_t STAGE = Sm::STAGE;
        const PrefixView pv{a.P, a.PT, a.PC};
        uint32_t tc = 0, staged = 0;
        int tab_tt = -1, my_d = 0, nd = 0; // mixed: the template tile of the warp's length tables
        for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x, tc++)
        {
            const int buf = tc & 1;
            const int tt = (int)(tile / ua.w_tiles);
            const uint32_t j0 = (uint32_t)(tile % ua.w_tiles) * TN;
            const float shift = tile_shift<MIXED>(a, j0);
            const int t = tt * TM + row;
            TemplParam p;
            bool valid = t < a.T;
            if (valid)
            {
                p = a.tp[t];
                valid = !MIXED || p.wcount > 0; // padding rows of mixed tiles
            }
            if (!valid)
            {
                p = TemplParam{};
                p.thr_ed = -kFltMax;
            }
            if (!MIXED)
            {
                // the window part of the bound once per window, with the maxima over the
                // tile's rows of its coefficients (all >= 0, so the maxima bound every row's):
                // each warp reduces its rows, the window terms are staged, and after the
                // barrier each thread folds the 8 warps' maxima into its window's eb
                const int wb = buf & (Sm::W2 - 1);
                const float c1 = warp_max_nonneg(valid, p.a1_main), c45 = warp_max_nonneg(valid, 2.0f * p.a4 + p.a5);
                const float c6 = warp_max_nonneg(valid, p.a6), c24 = warp_max_nonneg(valid, p.a2 + p.a4);
                if (lane == 0)
                    sm.coef[ew] = make_float4(c1, c45, c6, c24);
                const uint32_t j = j0 + et; // one window per epilogue thread
                float h;
                sm.win4[wb][et] = j < a.W ? win_terms(a.mean[j], a.inv[j], shift, h) : skip_terms(h);
                sm.win_h[wb][et] = h;
                mbar_arrive(&sm.win_ready[buf]);
                if (!mbar_wait_warp(&sm.win_ready[buf], (tc >> 1) & 1, sm.abort, ua.err, 7))
                    goto done;
                float4 cm = sm.coef[0];
#pragma unroll
                for (int w = 1; w < 8; w++)
                {
                    const float4 c = sm.coef[w];
                    cm = make_float4(fmaxf(cm.x, c.x), fmaxf(cm.y, c.y), fmaxf(cm.z, c.z), fmaxf(cm.w, c.w));
                }
                float4 wt = sm.win4[wb][et]; // each thread rewrites only its own window's entry
                wt.z = fmaf(cm.x, wt.z, fmaf(cm.y, wt.w, fmaf(cm.z, sm.win_h[wb][et], cm.w))); // eb (NaN: not searched)
                sm.win4[wb][et] = wt;
                mbar_arrive(&sm.eb_ready[buf]);
                if (!mbar_wait_warp(&sm.eb_ready[buf], (tc >> 1) & 1, sm.abort, ua.err, 8))
                    goto done;
            }
            // mixed: the distinct lengths of this warp's rows (at most 32), found while the
            // tile's MMAs run; my_d is the lane's entry. The tables depend only on the
            // template tile, so a warp keeps them while its next tiles have the same one.
            if (MIXED && tt != tab_tt)
            {
                tab_tt = tt;
                my_d = 0;
                nd = 0;
                __syncwarp(); // the previous tile's readers of the tables are done
                uint32_t pending = __ballot_sync(0xffffffffu, valid);
                while (pending != 0u)
                {
                    const int leader = __ffs(pending) - 1;
                    const int len = __shfl_sync(0xffffffffu, p.m, leader);
                    const bool mine = valid && p.m == len;
                    const uint32_t same = __ballot_sync(0xffffffffu, mine);
                    if (mine)
                        my_d = nd;
                    // bound coefficients of the length: maxima over its rows (all >= 0, so
                    // the float bit patterns order like the values)
                    const float c1 = warp_max_nonneg(mine, p.a1_main), c5 = warp_max_nonneg(mine, p.a5);
                    const float c6 = warp_max_nonneg(mine, p.a6);
                    const float cA = warp_max_nonneg(mine, 1.25f * (4.0f * (float)p.m + 2.0f * p.qs));
                    const float cB = warp_max_nonneg(mine, 2.5f * fabsf(p.s1));
                    if (lane == leader)
                    {
                        sm.wl_len[ew][nd] = len;
                        sm.wl_wc[ew][nd] = p.wcount; // a function of the length alone
                        sm.wl_inv[ew][nd] = p.inv_m;
                        sm.wl_fim[ew][nd] = (float)p.inv_m * (1.0f + 1.1920929e-07f);
                        sm.wl_c[ew][nd] = make_float4(c1, c5, c6, cA);
                        sm.wl_b[ew][nd] = cB;
                    }
                    nd++;
                    pending &= ~same;
                }
                __syncwarp();
            }
            if (!mbar_wait_warp(&sm.acc_full[buf], (tc >> 1) & 1, sm.abort, ua.err, 6))
                goto done;
            tc_fence_after();
            float umin = inf_f(), lmin = inf_f();
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * TN);
            if (MIXED)
            {
                // This warp's 128 windows of the tile (128 half .. + 127) in groups of G
                // windows, G x nd <= 256 table entries (G = 32 for up to 8 lengths):
                // phase A: statistics of each (window, distinct length of the warp) from the
                //   prefix sums at the window's start and end (the G lanes of a length read G
                //   consecutive windows; a lane's lengths share its window);
                // phase B: each lane's distances from its length's statistics, 8 windows
                //   per TMEM load, one candidate emission per group.
                const LaneTerms lt = lane_terms(p, valid);
                const int glog = nd <= 8 ? 5 : (nd <= 16 ? 4 : 3);
                const int G = 1 << glog;
                for (int c0 = 128 * half; c0 < 128 * half + 128; c0 += G)
                {
                    // item q = lane + 32 it is window i = lane mod G of the group and distinct
                    // length d = (lane >> glog) + it (32 >> glog): a lane's items share one
                    // window, so its start (prefix sums, first sample, constant run, block) is
                    // loaded once; its items go four at a time, the window ends loaded first,
                    // then the fast-path statistics of all four (prefix_stats_fast) as
                    // independent straight-line chains, then (rarely) the full bound for those
                    // that end in the next prefix block or are ill-conditioned
                    const int i = lane & (G - 1), d0 = lane >> glog, dstep = 32 >> glog;
                    const uint32_t j = j0 + (uint32_t)(c0 + i);
                    const uint64_t g = a.w0 + j;
                    const uint64_t b1 = g >> kPrefixBlockLog;
                    double2 qa = make_double2(0.0, 0.0);
                    float rv = kMissing;
                    uint16_t rn = 0xffffu;
                    double cen = 0.0, t2 = 0.0;
                    if (g < a.n)
                    {
                        qa = a.P[g];
                        rv = a.raw[g];
                        rn = a.run[g];
                        cen = a.PC[b1];
                        t2 = a.PT[b1].y;
                    }
                    const float cf = (float)cen;
                    const BlockBounds bb = block_bounds(t2);
#pragma unroll
                    for (int it0 = 0; it0 < 8; it0 += 4)
                    {
                        if (d0 + dstep * it0 >= nd)
                            break; // no length left for this lane (nothing in the loop is warp-collective)
                        double2 qb[4];
                        bool srch[4];
#pragma unroll
                        for (int k = 0; k < 4; k++)
                        {
                            const int d = d0 + dstep * (it0 + k); // < 32
                            const int len = sm.wl_len[ew][d];
                            srch[k] = d < nd && j < sm.wl_wc[ew][d] && rv != kMissing && rn < len;
                            qb[k] = make_double2(0.0, 0.0);
                            if (d < nd && j < sm.wl_wc[ew][d]) // then w0 + j + len <= n: both prefix entries exist
                                qb[k] = a.P[g + (uint64_t)len];
                        }
                        float4 r[4];
                        bool fast[4];
#pragma unroll
                        for (int k = 0; k < 4; k++)
                        {
                            const int d = d0 + dstep * (it0 + k);
                            const int len = sm.wl_len[ew][d];
                            float mu, iv, emu;
                            fast[k] = prefix_stats_fast(qa, qb[k], sm.wl_inv[ew][d], sm.wl_fim[ew][d], cf, bb, mu, iv,
                                                        emu) &&
                                      ((g + (uint64_t)len) >> kPrefixBlockLog) == b1;
                            r[k] = mixed_terms_fast(mu, iv, emu, shift, sm.wl_c[ew][d], sm.wl_b[ew][d]);
                        }
#pragma unroll
                        for (int k = 0; k < 4; k++)
                        {
                            const int d = d0 + dstep * (it0 + k);
                            if (srch[k] && !fast[k]) // two prefix blocks, or ill-conditioned: the full bound
                            {
                                const int len = sm.wl_len[ew][d];
                                WindowStats ws;
                                r[k] = window_prefix_stats(pv, qa, qb[k], g, len, sm.wl_inv[ew][d], ws) == 0
                                           ? mixed_terms(ws, shift, sm.wl_c[ew][d], sm.wl_b[ew][d])
                                           : make_float4(0.0f, 0.0f, inf_f(), 0.0f);
                            }
                            // not searched: NaN; statistics not trustworthy: E0 = +inf (d - e =
                            // -inf, exact re-scoring decides)
                            if (!srch[k])
                                r[k] = make_float4(0.0f, 0.0f, nan_f(), 0.0f);
                            if (d < nd)
                                sm.wst[ew][(d << glog) + (i ^ (d & 7))] = r[k];
                        }
                    }
                    __syncwarp();
                    uint32_t mask = 0;
                    const float4 *mine = &sm.wst[ew][my_d << glog];
                    for (int s8 = 0; s8 < G; s8 += 8)
                    {
                        float v[8];
                        tmem_ld8(taddr + c0 + s8, v);
#pragma unroll
                        for (int i = 0; i < 8; i++)
                        {
                            const float4 w = mine[(s8 + i) ^ (my_d & 7)];
                            pair_update(lt, v[i], w.x, w.y, w.z + lt.a2, s8 + i, mask, umin, lmin);
                        }
                        if (a.dbg_d != nullptr && valid)
                            for (int i = 0; i < 8; i++)
                            {
                                const float4 w = mine[(s8 + i) ^ (my_d & 7)];
                                if (w.x == 0.0f)
                                    continue; // not searched, or untrustworthy statistics
                                float dd, e;
                                pair_bound(lt, v[i], w.x, w.y, w.z + lt.a2, dd, e);
                                const size_t at = (size_t)t * a.W + j0 + c0 + s8 + i;
                                a.dbg_d[at] = dd;
                                a.dbg_e[at] = e;
                            }
                    }
                    __syncwarp(); // every lane has read the group's statistics
                    stage_emit<STAGE>(mask, lane, (uint32_t)t, j0 + c0, sm.stage[ew], staged, a.cand, a.cand_count,
                                      a.cand_cap);
                }
            }
            else
            {
                const int wb = buf & (Sm::W2 - 1);
                const LaneTerms lt = lane_terms(p, valid);
                // a warp whose rows are all kNN (or padding) needs only the minima, one whose
                // rows are all threshold rows only the mask
                const bool all_knn = __all_sync(0xffffffffu, !valid || p.mode == 1);
                const bool all_thr = __all_sync(0xffffffffu, !valid || p.mode != 1);
                for (int c = 8 * half; c < 8 * half + 8; c++) // this warp's 128 of the 256 columns
                {
                    float v[16];
                    tmem_ld16(taddr + c * 16, v);
                    uint32_t mask = 0;
                    if (all_knn)
                    {
#pragma unroll
                        for (int i = 0; i < 16; i++)
                        {
                            const float4 w = sm.win4[wb][c * 16 + i];
                            float d, e;
                            pair_bound(lt, v[i], w.x, w.y, w.z, d, e);
                            umin = fminf(umin, d + e);
                            lmin = fminf(lmin, d - e);
                        }
                    }
                    else if (all_thr)
                    {
#pragma unroll
                        for (int i = 0; i < 16; i++)
                        {
                            const float4 w = sm.win4[wb][c * 16 + i];
                            float d, e;
                            pair_bound(lt, v[i], w.x, w.y, w.z, d, e);
                            mask |= (d - e <= lt.thr ? 1u : 0u) << i;
                        }
                    }
                    else
                    {
#pragma unroll
                        for (int i = 0; i < 16; i++)
                        {
                            const float4 w = sm.win4[wb][c * 16 + i];
                            pair_update(lt, v[i], w.x, w.y, w.z, i, mask, umin, lmin);
                        }
                    }
                    if (a.dbg_d != nullptr && valid)
                        for (int i = 0; i < 16; i++)
                        {
                            const float4 w = sm.win4[wb][c * 16 + i];
                            if (w.x == 0.0f)
                                continue;
                            float dd, e;
                            pair_bound(lt, v[i], w.x, w.y, w.z, dd, e);
                            const size_t at = (size_t)t * a.W + j0 + c * 16 + i;
                            a.dbg_d[at] = dd;
                            a.dbg_e[at] = e;
                        }
                    if (!all_knn)
                        stage_emit<STAGE>(mask, lane, (uint32_t)t, j0 + c * 16, sm.stage[ew], staged, a.cand,
                                          a.cand_count, a.cand_cap);
                }
            }
            tc_fence_before();
            mbar_arrive(&sm.acc_empty[buf]);
            stage_flush(sm.stage[ew], staged, lane, a.cand, a.cand_count, a.cand_cap);
            if (valid && p.mode == 1 && (umin <= kFltMax || lmin == -inf_f()))
            {
                const size_t at = (size_t)t * a.nb + j0 / kBucket;
                atomicMin(&a.bmin_u[at], float_key(umin));
                atomicMin(&a.bmin_l[at], float_key(lmin));
            }
        }
    }
done:
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == 1)
    {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}


// ---- window-major variant ----------------------------------------------------------
//
// The same split-BF16 contraction with the roles of the operands exchanged: 128 windows
// on the MMA's M side (TMEM lanes) and NT templates on its N side (TMEM columns), for
// groups whose templates are too few per length for 128-row template tiles (each tile's
// K extent is its longest template, so a tile of mixed lengths wastes the difference).
// Column tiles of NT = 32, 64 or 128 templates of similar length keep that waste small.
//   A (windows): the Hankel strip, U[u][r][e] = split(x[j0 + k0 + 8u + r + e] - shift),
//     u < 128/8 + 64/8, described with SBO = LBO = 128 bytes as for the B operand of
//     k_scan_umma (the canonical K-major no-swizzle layout is the same for A and B).
//   B (templates, K-major): TMA tiles of NT rows x 64 samples, SWIZZLE_128B, hi and lo.
// Epilogue: a thread owns one window (its TMEM lane) and walks the tile's columns; the
// column's template is warp-uniform, so its constants come from shared memory (staged
// per tile) and mode branches do not diverge. Window statistics of each column's length
// come from the resident prefix sums (window_prefix_stats), with the window-end sums of 8
// columns loaded at once.

struct ColParam // the epilogue's constants of one template column
{
    double inv_m;
    float c_lin, s1, a1, a2, a3, a4, a5, a6, thr, qs;
    int m, mode;
    uint32_t wcount; // 0: padding column
    int pad;
};

constexpr int WM_M = 128;                        // windows per tile
constexpr int WM_STRIP = WM_M / 8 + KB / 8;      // 24 core matrices of 128 bytes
constexpr int WM_A_BYTES = WM_STRIP * 128;

template <int NT> struct SmemWM
{
    static constexpr int S = NT >= 128 ? 4 : (NT >= 64 ? 6 : 8);
    static constexpr int B_BYTES_T = NT * KB * 2;
    uint8_t b_hi[S][B_BYTES_T]; // 1024-byte aligned (swizzle atoms): NT * 128 is a multiple of 1024
    uint8_t b_lo[S][B_BYTES_T];
    uint8_t a_hi[S][WM_A_BYTES];
    uint8_t a_lo[S][WM_A_BYTES];
    ColParam cp[2][NT];
    Candidate stage[8][64];
    uint64_t full_a[S], full_b[S], empty[S];
    uint64_t acc_full[2], acc_empty[2], par_ready[2], drain;
    uint32_t tmem_base;
    int abort;
};

static_assert(sizeof(SmemWM<128>) + 1024 <= 227 * 1024, "shared memory of k_scan_wm<128>");
static_assert(sizeof(SmemWM<64>) + 1024 <= 227 * 1024, "shared memory of k_scan_wm<64>");
static_assert(sizeof(SmemWM<32>) + 1024 <= 227 * 1024, "shared memory of k_scan_wm<32>");

// Tile shift: the middle sample of the 128 windows (several lengths) or the mean of the
// middle window (one length).
template <bool MIXED> __device__ __forceinline__ float wm_shift(const ScanArgs &a, uint32_t j0)
{
    const uint32_t jm = min(j0 + WM_M / 2, a.W - 1);
    return MIXED ? a.x[a.w0 + jm] : a.mean[jm];
}

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_m128(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(WM_M >> 4) << 24);
}

template <int NT>
__device__ __forceinline__ void mma_n(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
                 "l"(a), "l"(b), "r"(idesc_m128(NT)), "r"(accumulate)
                 : "memory");
}

struct WmArgs
{
    ScanArgs a;
    int c_tiles, w_tiles, kblocks;
    int *err;
};

// MIXED: templates of several lengths, statistics from the prefix sums, K blocks per
// column tile (a.tiles); otherwise one length, the per-window statistics a.mean / a.inv
// of that length and a.m_pad / 64 K blocks everywhere.
template <int NT, bool MIXED>
__global__ void __launch_bounds__(THREADS, 1)
    k_scan_wm(const WmArgs wa, const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    using Sm = SmemWM<NT>;
    constexpr int STAGES = Sm::S;
    constexpr uint32_t COLS = (NT < 32 ? 32 : NT);
    Sm &sm = *reinterpret_cast<Sm *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const ScanArgs &a = wa.a;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long tiles = (long long)wa.c_tiles * wa.w_tiles;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < STAGES; s++)
        {
            mbar_init(&sm.full_a[s], 1);
            mbar_init(&sm.full_b[s], BUILDERS);
            mbar_init(&sm.empty[s], 1);
        }
        for (int b = 0; b < 2; b++)
        {
            mbar_init(&sm.acc_full[b], 1);
            mbar_init(&sm.acc_empty[b], EPI);
            mbar_init(&sm.par_ready[b], EPI);
        }
        mbar_init(&sm.drain, 1);
        sm.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&sm.tmem_base)),
                     "r"(2 * COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;

    if (warp == 0)
    {
        // ---- TMA producer: template column tiles (hi, lo) ----
        if (lane == 0)
        {
            uint32_t it = 0;
            for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x)
            {
                const int ct = (int)(tile / wa.w_tiles);
                const int kblocks = MIXED ? a.tiles[ct].kb : wa.kblocks;
                for (int kb = 0; kb < kblocks; kb++, it++)
                {
                    const int s = it % STAGES;
                    if (!mbar_wait(&sm.empty[s], ((it / STAGES) & 1) ^ 1, sm.abort, wa.err, 21))
                    {
                        for (uint32_t i = it > STAGES ? it - STAGES : 0; i < it; i++)
                            mbar_drain(&sm.full_a[i % STAGES], (i / STAGES) & 1);
                        goto done;
                    }
                    mbar_expect_tx(&sm.full_a[s], 2 * Sm::B_BYTES_T);
                    tma_load_2d(sm.b_hi[s], &map_hi, kb * KB, ct * NT, &sm.full_a[s]);
                    tma_load_2d(sm.b_lo[s], &map_lo, kb * KB, ct * NT, &sm.full_a[s]);
                }
            }
        }
    }
    else if (warp == 1)
    {
        // ---- MMA issuer ----
        if (lane == 0)
        {
            uint32_t it = 0, tc = 0;
            for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x, tc++)
            {
                const int buf = tc & 1;
                if (!mbar_wait(&sm.acc_empty[buf], ((tc >> 1) & 1) ^ 1, sm.abort, wa.err, 22))
                {
                    mma_commit(&sm.drain);
                    mbar_drain(&sm.drain, 0);
                    goto done;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(buf * COLS);
                const int kblocks = MIXED ? a.tiles[tile / wa.w_tiles].kb : wa.kblocks;
                for (int kb = 0; kb < kblocks; kb++, it++)
                {
                    const int s = it % STAGES;
                    const uint32_t ph = (it / STAGES) & 1;
                    if (!mbar_wait(&sm.full_a[s], ph, sm.abort, wa.err, 23) ||
                        !mbar_wait(&sm.full_b[s], ph, sm.abort, wa.err, 24))
                    {
                        mma_commit(&sm.drain);
                        mbar_drain(&sm.drain, 0);
                        goto done;
                    }
                    tc_fence_after();
                    const uint32_t ah = saddr(sm.a_hi[s]), al = saddr(sm.a_lo[s]);
                    const uint32_t bh = saddr(sm.b_hi[s]), bl = saddr(sm.b_lo[s]);
#pragma unroll
                    for (int kk = 0; kk < KB / 16; kk++)
                    {
                        const uint64_t dah = sdesc(ah + kk * 256, 128, 128, 0);
                        const uint64_t dal = sdesc(al + kk * 256, 128, 128, 0);
                        const uint64_t dbh = sdesc(bh + kk * 32, 16, 1024, 2);
                        const uint64_t dbl = sdesc(bl + kk * 32, 16, 1024, 2);
                        mma_n<NT>(d, dah, dbh, (kb | kk) != 0);
                        mma_n<NT>(d, dah, dbl, 1);
                        mma_n<NT>(d, dal, dbh, 1);
                    }
                    mma_commit(&sm.empty[s]);
                }
                mma_commit(&sm.acc_full[buf]);
            }
        }
    }
    else if (warp < 4)
    {
        // ---- strip builders (128 windows) ----
        const int tid = threadIdx.x - 64;
        uint32_t it = 0;
        for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x)
        {
            const uint32_t j0 = (uint32_t)(tile % wa.w_tiles) * WM_M;
            const float shift = wm_shift<MIXED>(a, j0);
            const float *xw = a.x + a.w0 + j0;
            const int kblocks = MIXED ? a.tiles[tile / wa.w_tiles].kb : wa.kblocks;
            for (int kb = 0; kb < kblocks; kb++, it++)
            {
                const int s = it % STAGES;
                if (!mbar_wait(&sm.empty[s], ((it / STAGES) & 1) ^ 1, sm.abort, wa.err, 25))
                    goto done;
                const float *xs = xw + kb * KB;
                for (int row = tid; row < WM_STRIP * 8; row += BUILDERS)
                {
                    const int u = row >> 3, r = row & 7;
                    float v[8], h[8], l[8];
#pragma unroll
                    for (int e = 0; e < 8; e++)
                        v[e] = xs[8 * u + r + e] - shift;
#pragma unroll
                    for (int e = 0; e < 8; e++)
                    {
                        h[e] = __bfloat162float(__float2bfloat16_rn(v[e]));
                        l[e] = v[e] - h[e];
                    }
                    uint4 hv, lv;
                    hv.x = pack_bf16(h[0], h[1]);
                    hv.y = pack_bf16(h[2], h[3]);
                    hv.z = pack_bf16(h[4], h[5]);
                    hv.w = pack_bf16(h[6], h[7]);
                    lv.x = pack_bf16(l[0], l[1]);
                    lv.y = pack_bf16(l[2], l[3]);
                    lv.z = pack_bf16(l[4], l[5]);
                    lv.w = pack_bf16(l[6], l[7]);
                    *reinterpret_cast<uint4 *>(&sm.a_hi[s][u * 128 + r * 16]) = hv;
                    *reinterpret_cast<uint4 *>(&sm.a_lo[s][u * 128 + r * 16]) = lv;
                }
                fence_proxy_async();
                mbar_arrive(&sm.full_b[s]);
            }
        }
    }
    else
    {
        // ---- epilogue (8 warps): warp (quarter, half) holds windows 32 quarter + lane and
        // the half of the tile's columns ----
        const int quarter = warp & 3;
        const int ew = warp - 4;
        const int half = ew >> 2;
        const int et = threadIdx.x - 128;
        const PrefixView pv{a.P, a.PT, a.PC};
        uint32_t tc = 0, staged = 0;
        for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x, tc++)
        {
            const int buf = tc & 1;
            const int ct = (int)(tile / wa.w_tiles);
            const uint32_t j0 = (uint32_t)(tile % wa.w_tiles) * WM_M;
            if (et < NT)
            {
                const int t = ct * NT + et;
                ColParam c{};
                if (t < a.T)
                {
                    const TemplParam &p = a.tp[t];
                    c.inv_m = p.inv_m;
                    c.c_lin = p.c_lin;
                    c.s1 = p.s1;
                    c.a1 = p.a1_main;
                    c.a2 = p.a2;
                    c.a3 = p.a3;
                    c.a4 = p.a4;
                    c.a5 = p.a5;
                    c.a6 = p.a6;
                    c.thr = p.thr_ed;
                    c.qs = p.qs;
                    c.m = p.m;
                    c.mode = p.mode;
                    c.wcount = MIXED ? p.wcount : 1u; // one length: every real row is searched
                }
                else
                {
                    c.m = 1;
                    c.thr = -kFltMax;
                }
                sm.cp[buf][et] = c;
            }
            mbar_arrive(&sm.par_ready[buf]);
            if (!mbar_wait_warp(&sm.par_ready[buf], (tc >> 1) & 1, sm.abort, wa.err, 27))
                goto done;
            const uint32_t j = j0 + (uint32_t)(quarter * 32 + lane);
            const bool in = j < a.W;
            double2 pj = make_double2(0.0, 0.0);
            uint32_t runj = 0;
            bool miss = !in;
            float wmean = 0.0f, winv = 0.0f; // one length: the window's statistics (inv 0: not searched)
            if (MIXED)
            {
                if (in)
                {
                    pj = a.P[a.w0 + j];
                    runj = a.run[a.w0 + j];
                    miss = a.raw[a.w0 + j] == kMissing;
                }
            }
            else if (in)
            {
                wmean = a.mean[j];
                winv = a.inv[j];
                miss = winv == 0.0f;
            }
            // mixed: the window's prefix block, the block's centre and its fast-path error bounds
            const uint64_t jb = (a.w0 + j) >> kPrefixBlockLog;
            const float jcf = MIXED && in ? (float)a.PC[jb] : 0.0f;
            const BlockBounds jbb = block_bounds(MIXED && in ? a.PT[jb].y : 0.0);
            const float shift = wm_shift<MIXED>(a, j0);
            const size_t bucket = j0 / kBucket;
            if (!mbar_wait_warp(&sm.acc_full[buf], (tc >> 1) & 1, sm.abort, wa.err, 26))
                goto done;
            tc_fence_after();
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * COLS);
            for (int g = half * (NT / 2); g < (half + 1) * (NT / 2); g += 8)
            {
                double2 pe[8];
#pragma unroll
                for (int i = 0; i < 8; i++)
                {
                    const ColParam &c = sm.cp[buf][g + i];
                    const bool ok = MIXED && !miss && j < c.wcount && runj < (uint32_t)c.m;
                    pe[i] = ok ? a.P[a.w0 + j + (uint32_t)c.m] : make_double2(0.0, 0.0);
                }
                float v[8];
                tmem_ld8(taddr + g, v);
#pragma unroll
                for (int h4 = 0; h4 < 8; h4 += 4)
                {
                    // mixed: the statistics of the window for four columns' lengths, as four
                    // independent fast-path evaluations (prefix_stats_fast), then (rarely) the
                    // full bound for those whose window ends in the next prefix block or is
                    // ill-conditioned
                    WindowStats wsv[4];
                    int wst[4];
                    if (MIXED)
                    {
#pragma unroll
                        for (int k = 0; k < 4; k++)
                        {
                            const ColParam &c = sm.cp[buf][g + h4 + k];
                            const bool fast =
                                prefix_stats_fast(pj, pe[h4 + k], c.inv_m, (float)c.inv_m * (1.0f + 1.1920929e-07f), jcf,
                                                  jbb, wsv[k].mu, wsv[k].iv, wsv[k].e_mu) &&
                                ((a.w0 + j + (uint64_t)c.m) >> kPrefixBlockLog) == jb;
                            wsv[k].rel_sd = kFastRelSd;
                            wst[k] = fast ? 0 : 1;
                        }
#pragma unroll
                        for (int k = 0; k < 4; k++)
                        {
                            const ColParam &c = sm.cp[buf][g + h4 + k];
                            const bool ok = !miss && j < c.wcount && runj < (uint32_t)c.m;
                            if (ok && wst[k] != 0) // two prefix blocks, or ill-conditioned: the full bound
                                wst[k] = window_prefix_stats(pv, pj, pe[h4 + k], a.w0 + j, c.m, c.inv_m, wsv[k]);
                        }
                    }
#pragma unroll
                    for (int k = 0; k < 4; k++)
                    {
                        const int i = h4 + k;
                        const ColParam &c = sm.cp[buf][g + i];
                        const uint32_t t = (uint32_t)(ct * NT + g + i);
                        const bool ok = MIXED ? (!miss && j < c.wcount && runj < (uint32_t)c.m) : (!miss && c.wcount > 0);
                        bool hit = false;
                        float up = inf_f(), lo = inf_f();
                        if (!MIXED && ok)
                        {
                            const float ms = wmean - shift;
                            const float cross = (v[i] - ms * c.s1) * winv;
                            const float dd = c.c_lin - 2.0f * cross;
                            const float r = ms * winv, r0 = wmean * winv;
                            const float e = c.a1 * sqrtf(1.0f + r * r) + c.a2 + c.a3 * fmaxf(dd, 0.0f) +
                                            c.a4 * (1.0f + 2.0f * r0 * r0) + c.a5 * r0 * r0 +
                                            c.a6 * (fabsf(wmean) + fabsf(shift)) * winv;
                            if (a.dbg_d != nullptr)
                            {
                                a.dbg_d[(size_t)t * a.W + j] = dd;
                                a.dbg_e[(size_t)t * a.W + j] = e;
                            }
                            up = dd + e;
                            lo = dd - e;
                            hit = lo <= c.thr;
                        }
                        else if (ok)
                        {
                            const WindowStats &ws = wsv[k];
                            if (wst[k] == 0)
                            {
                                const float ms = ws.mu - shift;
                                const float cross = (v[i] - ms * c.s1) * ws.iv;
                                const float dd = c.c_lin - 2.0f * cross;
                                const float r = ms * ws.iv, r0 = ws.mu * ws.iv;
                                const float e = c.a1 * sqrtf(1.0f + r * r) + c.a2 + c.a3 * fmaxf(dd, 0.0f) +
                                                c.a5 * r0 * r0 + c.a6 * (fabsf(ws.mu) + fabsf(shift)) * ws.iv +
                                                stats_error(ws, c.m, c.qs, c.s1);
                                if (a.dbg_d != nullptr)
                                {
                                    a.dbg_d[(size_t)t * a.W + j] = dd;
                                    a.dbg_e[(size_t)t * a.W + j] = e;
                                }
                                up = dd + e;
                                lo = dd - e;
                                hit = lo <= c.thr;
                            }
                            else
                            {
                                lo = -inf_f(); // statistics not trustworthy: exact re-scoring decides
                                hit = true;
                            }
                        }
                        if (c.mode == 1) // kNN: bucket minima over the warp's 32 windows
                        {
                            const uint32_t ku = __reduce_min_sync(0xffffffffu, float_key(up));
                            const uint32_t kl = __reduce_min_sync(0xffffffffu, float_key(lo));
                            if (lane == 0 && (ku != float_key(inf_f()) || kl != float_key(inf_f())))
                            {
                                atomicMin(&a.bmin_u[(size_t)t * a.nb + bucket], ku);
                                atomicMin(&a.bmin_l[(size_t)t * a.nb + bucket], kl);
                            }
                        }
                        else
                            stage_emit_lane<64>(hit, lane, t, j, sm.stage[ew], staged, a.cand, a.cand_count, a.cand_cap);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&sm.acc_empty[buf]);
            stage_flush(sm.stage[ew], staged, lane, a.cand, a.cand_count, a.cand_cap);
        }
    }
done:
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == 1)
    {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * COLS));
    }
}

// ---- host side -------------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
    }();
    return fn;
}

// BF16 row-major [rows][cols] operand, boxes of 64 samples x box_rows rows, 128-byte swizzle.
bool make_map(CUtensorMap *map, const void *base, int rows, int cols, int box_rows = TM)
{
    auto fn = encode_fn();
    if (fn == nullptr)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)KB, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

} // namespace umma

bool umma_supported(int m, int T, uint64_t W)
{
    (void)m;
    (void)T;
    (void)W;
    static int ok = -1;
    if (ok < 0)
    {
        int dev = 0, major = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        ok = (major == 10 && umma::encode_fn() != nullptr) ? 1 : 0;
    }
    return ok == 1;
}

cudaError_t launch_scan_umma(const ScanArgs &a, cudaStream_t s)
{
    using namespace umma;
    if (a.q_hi == nullptr || a.q_lo == nullptr || a.err == nullptr)
        return cudaErrorInvalidValue;
    const bool mixed = a.tiles != nullptr;
    if (mixed && (a.P == nullptr || a.PT == nullptr || a.PC == nullptr || a.run == nullptr || a.raw == nullptr))
        return cudaErrorInvalidValue;
    const int stride = mixed ? a.k_stride : a.m_pad;
    CUtensorMap mh, ml;
    if (!make_map(&mh, a.q_hi, a.t_rows, stride) || !make_map(&ml, a.q_lo, a.t_rows, stride))
        return cudaErrorInvalidValue;
    UmmaArgs ua;
    ua.a = a;
    ua.t_tiles = (a.T + TM - 1) / TM;
    ua.w_tiles = (int)((a.W + TN - 1) / TN);
    ua.kblocks = a.m_pad / KB;
    ua.err = a.err;
    const size_t smem = (mixed ? sizeof(SmemT<true>) : sizeof(SmemT<false>)) + 1024;
    static const cudaError_t attr = [] {
        cudaError_t e = cudaFuncSetAttribute(k_scan_umma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(sizeof(SmemT<false>) + 1024));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_scan_umma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(sizeof(SmemT<true>) + 1024));
        return e;
    }();
    if (attr != cudaSuccess)
        return attr;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (long long)ua.t_tiles * ua.w_tiles;
    const int grid = (int)std::min<long long>(tiles, sms);
    if (mixed)
        k_scan_umma<true><<<grid, THREADS, smem, s>>>(ua, mh, ml);
    else
        k_scan_umma<false><<<grid, THREADS, smem, s>>>(ua, mh, ml);
    return cudaGetLastError();
}

// Window-major contraction in column tiles of a.col_tile templates: a mixed-length group
// (a.tiles: one TileInfo per column tile, K blocks only; statistics from the prefix sums)
// or, when a.tiles is null, one length (a.mean / a.inv, a.m_pad samples).
template <int NT> static cudaError_t wm_attr()
{
    using namespace umma;
    cudaError_t e = cudaFuncSetAttribute(k_scan_wm<NT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sizeof(SmemWM<NT>) + 1024));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_scan_wm<NT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(SmemWM<NT>) + 1024));
    return e;
}

template <int NT>
static void wm_launch(bool mixed, int grid, const umma::WmArgs &wa, const CUtensorMap &mh, const CUtensorMap &ml,
                      cudaStream_t s)
{
    using namespace umma;
    if (mixed)
        k_scan_wm<NT, true><<<grid, THREADS, sizeof(SmemWM<NT>) + 1024, s>>>(wa, mh, ml);
    else
        k_scan_wm<NT, false><<<grid, THREADS, sizeof(SmemWM<NT>) + 1024, s>>>(wa, mh, ml);
}

cudaError_t launch_scan_wm(const ScanArgs &a, cudaStream_t s)
{
    using namespace umma;
    const int NT = a.col_tile;
    const bool mixed = a.tiles != nullptr;
    if ((NT != 32 && NT != 64 && NT != 128) || a.q_hi == nullptr || a.q_lo == nullptr || a.err == nullptr ||
        a.t_rows % NT != 0)
        return cudaErrorInvalidValue;
    if (mixed ? (a.P == nullptr || a.PT == nullptr || a.PC == nullptr || a.run == nullptr || a.raw == nullptr)
              : (a.mean == nullptr || a.inv == nullptr))
        return cudaErrorInvalidValue;
    const int stride = mixed ? a.k_stride : a.m_pad;
    CUtensorMap mh, ml;
    if (!make_map(&mh, a.q_hi, a.t_rows, stride, NT) || !make_map(&ml, a.q_lo, a.t_rows, stride, NT))
        return cudaErrorInvalidValue;
    WmArgs wa;
    wa.a = a;
    wa.c_tiles = a.t_rows / NT;
    wa.w_tiles = (int)((a.W + WM_M - 1) / WM_M);
    wa.kblocks = a.m_pad / KB;
    wa.err = a.err;
    static const cudaError_t attr = [] {
        cudaError_t e = wm_attr<32>();
        if (e == cudaSuccess)
            e = wm_attr<64>();
        if (e == cudaSuccess)
            e = wm_attr<128>();
        return e;
    }();
    if (attr != cudaSuccess)
        return attr;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (long long)wa.c_tiles * wa.w_tiles;
    const int grid = (int)std::min<long long>(tiles, sms);
    if (NT == 32)
        wm_launch<32>(mixed, grid, wa, mh, ml, s);
    else if (NT == 64)
        wm_launch<64>(mixed, grid, wa, mh, ml, s);
    else
        wm_launch<128>(mixed, grid, wa, mh, ml, s);
    return cudaGetLastError();
}

} // namespace tmb
