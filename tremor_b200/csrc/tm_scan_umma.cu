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
// Warp roles (256 threads): warp 0 TMA producer, warp 1 TMEM owner + MMA issuer,
// warps 2-3 strip builders, warps 4-7 epilogue (TMEM lane quarter = warp % 4).
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
constexpr int STAGES = 4;
constexpr int STRIP_CHUNKS = TN / 8 + KB / 8; // 40 core matrices of 128 bytes
constexpr int A_BYTES = TM * KB * 2;          // 16 KiB per half
constexpr int B_BYTES = STRIP_CHUNKS * 128;   // 5 KiB per half
constexpr int THREADS = 256;
constexpr int BUILDERS = 64;
constexpr uint32_t TMEM_COLS = 2 * TN;
constexpr long long TIMEOUT_CYCLES = 4000000000ll; // ~2 s at 2 GHz

struct Smem
{
    uint8_t a_hi[STAGES][A_BYTES]; // 1024-byte aligned (swizzle atoms)
    uint8_t a_lo[STAGES][A_BYTES];
    uint8_t b_hi[STAGES][B_BYTES];
    uint8_t b_lo[STAGES][B_BYTES];
    float win_mean[2][TN];
    float win_inv[2][TN];
    double2 win_p[2][TN];      // mixed-length tiles: prefix sums at each window start
    uint16_t win_run[2][TN];   //   constant-run length at each window start
    uint8_t win_miss[2][TN];   //   first sample missing
    uint64_t full_a[STAGES], full_b[STAGES], empty[STAGES];
    uint64_t acc_full[2], acc_empty[2], win_ready[2], drain;
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
// Bounded wait: false on timeout or when another role aborted (the CTA then unwinds).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, Smem &sm, int *err, int where)
{
    if (mbar_try(bar, parity))
        return true;
    const long long t0 = clock64();
    while (true)
    {
        if (mbar_try(bar, parity))
            return true;
        if (*(volatile int *)&sm.abort)
            return false;
        if (clock64() - t0 > TIMEOUT_CYCLES)
        {
            *(volatile int *)&sm.abort = 1;
            atomicExch(err, 1000 + where);
            return false;
        }
    }
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

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b); // .x = a (low half), .y = b
    return *reinterpret_cast<const uint32_t *>(&h);
}

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

template <bool MIXED>
__global__ void __launch_bounds__(THREADS, 1)
    k_scan_umma(const UmmaArgs ua, const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    Smem &sm = *reinterpret_cast<Smem *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
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
            mbar_init(&sm.acc_empty[b], 128);
            mbar_init(&sm.win_ready[b], 128);
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
                const int kblocks = MIXED ? a.tile_kb[tt] : ua.kblocks;
                for (int kb = 0; kb < kblocks; kb++, it++)
                {
                    const int s = it % STAGES;
                    if (!mbar_wait(&sm.empty[s], ((it / STAGES) & 1) ^ 1, sm, ua.err, 1))
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
                if (!mbar_wait(&sm.acc_empty[buf], ((tc >> 1) & 1) ^ 1, sm, ua.err, 2))
                {
                    mma_commit(&sm.drain);
                    mbar_drain(&sm.drain, 0);
                    goto done;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(buf * TN);
                const int kblocks = MIXED ? a.tile_kb[tile / ua.w_tiles] : ua.kblocks;
                for (int kb = 0; kb < kblocks; kb++, it++)
                {
                    const int s = it % STAGES;
                    const uint32_t ph = (it / STAGES) & 1;
                    if (!mbar_wait(&sm.full_a[s], ph, sm, ua.err, 3) || !mbar_wait(&sm.full_b[s], ph, sm, ua.err, 4))
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
            const int kblocks = MIXED ? a.tile_kb[tile / ua.w_tiles] : ua.kblocks;
            for (int kb = 0; kb < kblocks; kb++, it++)
            {
                const int s = it % STAGES;
                if (!mbar_wait(&sm.empty[s], ((it / STAGES) & 1) ^ 1, sm, ua.err, 5))
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
        // ---- epilogue: TMEM -> distances, bounds, candidates / bucket minima ----
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane; // TMEM lane = template within the tile
        const int et = threadIdx.x - 128;    // 0..127
        uint32_t tc = 0;
        for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x, tc++)
        {
            const int buf = tc & 1;
            const int tt = (int)(tile / ua.w_tiles);
            const uint32_t j0 = (uint32_t)(tile % ua.w_tiles) * TN;
            for (int i = et; i < TN; i += 128)
            {
                const uint32_t j = j0 + i;
                if (MIXED)
                {
                    const bool in = j < a.W;
                    sm.win_p[buf][i] = in ? a.P[a.w0 + j] : make_double2(0.0, 0.0);
                    sm.win_run[buf][i] = in ? a.run[a.w0 + j] : (uint16_t)65535;
                    sm.win_miss[buf][i] = in ? (uint8_t)(a.raw[a.w0 + j] == kMissing) : (uint8_t)1;
                }
                else
                {
                    sm.win_mean[buf][i] = j < a.W ? a.mean[j] : 0.0f;
                    sm.win_inv[buf][i] = j < a.W ? a.inv[j] : 0.0f;
                }
            }
            mbar_arrive(&sm.win_ready[buf]);
            if (!mbar_wait(&sm.win_ready[buf], (tc >> 1) & 1, sm, ua.err, 7))
                goto done;
            const float shift = tile_shift<MIXED>(a, j0);
            const int t = tt * TM + row;
            const bool valid = t < a.T;
            TemplParam p;
            if (valid)
                p = a.tp[t];
            else
            {
                p.mode = 0;
                p.thr_ed = -kFltMax;
            }
            if (!mbar_wait(&sm.acc_full[buf], (tc >> 1) & 1, sm, ua.err, 6))
                goto done;
            tc_fence_after();
            float umin = inf_f(), lmin = inf_f();
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * TN);
            for (int c = 0; c < TN / 16; c++)
            {
                float v[16];
                tmem_ld16(taddr + c * 16, v);
                uint32_t mask = 0;
                if (valid && MIXED)
                {
#pragma unroll
                    for (int i = 0; i < 16; i++)
                    {
                        const int ci = c * 16 + i;
                        const uint32_t j = j0 + ci;
                        if (j >= p.wcount || sm.win_miss[buf][ci] || sm.win_run[buf][ci] >= p.m)
                            continue; // beyond this template's windows, missing first sample, constant
                        WindowStats ws;
                        if (prefix_stats(sm.win_p[buf][ci], a.P[a.w0 + j + p.m], a.w0 + j, p.m, p.inv_m, a.center,
                                         p.qs, p.s1, ws) != 0)
                        {
                            // statistics not trustworthy: the exact re-scoring decides this window
                            if (p.mode == 1)
                                lmin = -inf_f();
                            else
                                mask |= 1u << i;
                            continue;
                        }
                        float dd, e;
                        fast_distance_mixed(p, p.a1_main, v[i], ws.mu, ws.iv, shift, ws.estat, dd, e);
                        if (a.dbg_d != nullptr)
                        {
                            const size_t at = (size_t)t * a.W + j;
                            a.dbg_d[at] = dd;
                            a.dbg_e[at] = e;
                        }
                        const float lo = dd - e;
                        if (p.mode == 1)
                        {
                            umin = fminf(umin, dd + e);
                            lmin = fminf(lmin, lo);
                        }
                        else if (lo <= p.thr_ed)
                            mask |= 1u << i;
                    }
                }
                else if (valid)
                {
#pragma unroll
                    for (int i = 0; i < 16; i++)
                    {
                        const float iv = sm.win_inv[buf][c * 16 + i];
                        if (iv == 0.0f)
                            continue;
                        float dd, e;
                        fast_distance(p, p.a1_main, v[i], sm.win_mean[buf][c * 16 + i], iv, shift, dd, e);
                        if (a.dbg_d != nullptr)
                        {
                            const size_t at = (size_t)t * a.W + j0 + c * 16 + i;
                            a.dbg_d[at] = dd;
                            a.dbg_e[at] = e;
                        }
                        const float lo = dd - e;
                        if (p.mode == 1)
                        {
                            umin = fminf(umin, dd + e);
                            lmin = fminf(lmin, lo);
                        }
                        else if (lo <= p.thr_ed)
                            mask |= 1u << i;
                    }
                }
                emit_candidates(mask, lane, (uint32_t)t, j0 + c * 16, a.cand, a.cand_count, a.cand_cap);
            }
            tc_fence_before();
            mbar_arrive(&sm.acc_empty[buf]);
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

// ---- host side -------------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (fn == nullptr)
    {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

bool make_map(CUtensorMap *map, const void *base, int rows, int cols)
{
    auto fn = encode_fn();
    if (fn == nullptr)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)KB, (cuuint32_t)TM};
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
    const bool mixed = a.tile_kb != nullptr;
    if (mixed && (a.P == nullptr || a.run == nullptr || a.raw == nullptr))
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
    const size_t smem = sizeof(Smem) + 1024;
    static bool attr = false;
    if (!attr)
    {
        cudaError_t e = cudaFuncSetAttribute(k_scan_umma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_scan_umma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return e;
        attr = true;
    }
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

} // namespace tmb
