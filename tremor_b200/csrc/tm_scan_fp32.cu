// Plain FP32 contraction: the sliding dot products of a tile of templates against a
// tile of windows on the CUDA cores, with the distance epilogue fused.
//
// For template t (z-normalised, q) and window j (raw x, statistics mu_j, sigma_j)
//     ED^2 = sum q^2 + m - 2 (sum_i q_i (x_{j+i} - s) - (mu_j - s) sum q) / sigma_j
// (the identity of fft_fallback.hpp:112), with a per-tile shift s that keeps the
// products small when the waveform has an offset. Each result carries a rigorous
// bound E on its distance to the reference's FP32 distance (fast_distance in
// tm_epilogue.cuh), so the
// epilogue can decide, without the reference arithmetic, which windows are certainly
// out of an answer set: threshold requests emit every window with d - E <= the
// threshold distance; kNN requests record per 2048-window bucket the smallest d + E
// and d - E, from which the kNN bound is selected afterwards (tm_select.cu).
//
// Tile: 256 windows x 64 templates per CTA, 8 warps; a warp owns 8 templates and a
// lane 8 consecutive windows (64 FP32 accumulators). K advances in stages of 64
// samples, three buffers deep with cp.async (one barrier per stage), the tile's shift
// subtracted as the samples are read into registers. The stage's waveform slice is stored with 4
// floats of padding after every 32 (xpos), so that the float4 loads of a quarter warp
// (lanes 8 floats apart) fall in distinct shared-memory banks; a float4 never straddles
// a pad because the loads start at multiples of 4 floats.
#include "tm_internal.cuh"
#include "tm_epilogue.cuh"

namespace tmb {

constexpr int F_WIN = 256, F_TPL = 64, F_THREADS = 256;
// per stage of K samples (64, or 128 when the padded length allows: half the barriers):
// the waveform slice (F_XS floats, stored with their padding) and the templates' slices
template <int K> struct FStage
{
    static constexpr int XS = F_WIN + K + 16;
    static constexpr int XS_PAD = XS + ((XS + 31) >> 5) * 4;
};

__device__ __forceinline__ int xpos(int i) { return i + ((i >> 5) << 2); }

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// Two FP32 values in one 64-bit register pair, and the packed FMA of sm_100 on such pairs:
// each half is an ordinary round-to-nearest fmaf, one instruction for two.
__device__ __forceinline__ uint64_t f2pack(float lo, float hi)
{
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2unpack(uint64_t v, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ void fma2(uint64_t &acc, uint64_t a, uint64_t b)
{
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(a), "l"(b));
}
template <int N> __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Three operand buffers (dynamic shared memory): stage st + 2 is loaded into the buffer
// that stage st - 1 used, so one barrier per stage both publishes stage st and retires
// stage st - 1.
constexpr int F_BUFS = 3;
template <int K> constexpr size_t f_smem()
{
    return sizeof(float) * (size_t)F_BUFS * (FStage<K>::XS_PAD + F_TPL * K);
}

template <int F_K>
__global__ void __launch_bounds__(F_THREADS, 2) k_scan_fp32(ScanArgs a)
{
    constexpr int F_XS = FStage<F_K>::XS, F_XS_PAD = FStage<F_K>::XS_PAD;
    extern __shared__ __align__(16) float fsm[];
    float(*xs)[F_XS_PAD] = reinterpret_cast<float(*)[F_XS_PAD]>(fsm);
    float(*qs)[F_K][F_TPL] = reinterpret_cast<float(*)[F_K][F_TPL]>(fsm + F_BUFS * F_XS_PAD);
    __shared__ TemplParam tps[F_TPL];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile_j = blockIdx.x * F_WIN;
    const int tile_t = blockIdx.y * F_TPL;
    if (tid < F_TPL)
        tps[tid] = a.tp[tile_t + tid];
    const uint32_t jmid = min(tile_j + F_WIN / 2, a.W - 1);
    const float shift = a.mean[jmid];
    const float *xg = a.x + a.w0 + tile_j;
    const float *qg = a.qt + (size_t)tile_t * a.m_pad; // the tile's templates, [k][64]

    auto load_stage = [&](int buf, int k0) {
        for (int i = tid; i < F_XS; i += F_THREADS)
            cp_async4(&xs[buf][xpos(i)], xg + k0 + i);
        for (int i = tid; i < F_TPL * F_K / 4; i += F_THREADS)
            cp_async16(&qs[buf][0][0] + i * 4, qg + (size_t)k0 * F_TPL + i * 4);
        cp_commit();
    };

    // acc2[w][p]: the products of window 8 lane + w with templates 8 warp + 2p and + 2p + 1
    uint64_t acc2[8][4];
#pragma unroll
    for (int w = 0; w < 8; w++)
#pragma unroll
        for (int p2 = 0; p2 < 4; p2++)
            acc2[w][p2] = 0ull;

    const int stages = a.m_pad / F_K;
    load_stage(0, 0);
    if (stages > 1)
        load_stage(1, F_K);
    for (int st = 0; st < stages; st++)
    {
        const int cur = st % F_BUFS;
        if (st + 1 < stages)
            cp_wait<1>(); // this thread's copies of stage st have landed (st + 1 may be in flight)
        else
            cp_wait<0>();
        __syncthreads(); // stage st visible to all; every warp is done with stage st - 1
        if (st + 2 < stages)
            load_stage((st + 2) % F_BUFS, (st + 2) * F_K);
        const float *xw = &xs[cur][0];
        const float *qw = &qs[cur][0][8 * warp];
#pragma unroll 4
        for (int kk = 0; kk < F_K; kk += 4)
        {
            const int x0 = 8 * lane + kk;
            const float4 xa = *reinterpret_cast<const float4 *>(xw + xpos(x0));
            const float4 xb = *reinterpret_cast<const float4 *>(xw + xpos(x0 + 4));
            const float4 xc = *reinterpret_cast<const float4 *>(xw + xpos(x0 + 8));
            // the tile's shift, subtracted in registers (the same float subtraction for every
            // use of a sample)
            const float xr[12] = {xa.x - shift, xa.y - shift, xa.z - shift, xa.w - shift,
                                  xb.x - shift, xb.y - shift, xb.z - shift, xb.w - shift,
                                  xc.x - shift, xc.y - shift, xc.z - shift, xc.w - shift};
            // sample kk + i of the warp's 8 templates (two broadcast float4 loads), as 4 pairs;
            // each accumulator takes its products in k order, as one fmaf each
#pragma unroll
            for (int i = 0; i < 4; i++)
            {
                const float4 qa = *reinterpret_cast<const float4 *>(qw + (kk + i) * F_TPL);
                const float4 qb = *reinterpret_cast<const float4 *>(qw + (kk + i) * F_TPL + 4);
                const uint64_t q2[4] = {f2pack(qa.x, qa.y), f2pack(qa.z, qa.w), f2pack(qb.x, qb.y),
                                        f2pack(qb.z, qb.w)};
#pragma unroll
                for (int w = 0; w < 8; w++)
                {
                    const uint64_t x2 = f2pack(xr[w + i], xr[w + i]);
#pragma unroll
                    for (int p2 = 0; p2 < 4; p2++)
                        fma2(acc2[w][p2], x2, q2[p2]);
                }
            }
        }
    }
    float acc[8][8];
#pragma unroll
    for (int w = 0; w < 8; w++)
#pragma unroll
        for (int p2 = 0; p2 < 4; p2++)
            f2unpack(acc2[w][p2], acc[w][2 * p2], acc[w][2 * p2 + 1]);

    // ---- fused epilogue ----
    const uint32_t j0 = tile_j + 8 * lane;
    float mu[8], iv[8];
#pragma unroll
    for (int w = 0; w < 8; w++)
    {
        const uint32_t j = j0 + w;
        mu[w] = j < a.W ? a.mean[j] : 0.0f;
        iv[w] = j < a.W ? a.inv[j] : 0.0f;
    }
    const uint32_t bucket = tile_j / kBucket;
#pragma unroll
    for (int tt = 0; tt < 8; tt++)
    {
        const int tl = 8 * warp + tt;
        const TemplParam &p = tps[tl];
        const int t = tile_t + tl;
        if (t >= a.T)
            break; // warp-uniform
        float umin = inf_f(), lmin = inf_f();
        uint32_t emit_mask = 0;
#pragma unroll
        for (int w = 0; w < 8; w++)
        {
            if (iv[w] == 0.0f)
                continue; // excluded window (beyond range, missing start, degenerate)
            float d, e;
            fast_distance(p, p.a1_main, acc[w][tt], mu[w], iv[w], shift, d, e);
            if (a.dbg_d != nullptr)
            {
                a.dbg_d[(size_t)t * a.W + j0 + w] = d;
                a.dbg_e[(size_t)t * a.W + j0 + w] = e;
            }
            const float lo = d - e, hi = d + e;
            if (p.mode == 1)
            {
                umin = fminf(umin, hi);
                lmin = fminf(lmin, lo);
            }
            else if (lo <= p.thr_ed)
                emit_mask |= 1u << w;
        }
        if (p.mode == 1)
        {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
            {
                umin = fminf(umin, __shfl_xor_sync(0xffffffffu, umin, off));
                lmin = fminf(lmin, __shfl_xor_sync(0xffffffffu, lmin, off));
            }
            if (lane == 0 && umin <= kFltMax)
            {
                atomicMin(&a.bmin_u[(size_t)t * a.nb + bucket], float_key(umin));
                atomicMin(&a.bmin_l[(size_t)t * a.nb + bucket], float_key(lmin));
            }
        }
        else
            emit_candidates(emit_mask, lane, (uint32_t)t, j0, a.cand, a.cand_count, a.cand_cap);
    }
}

// The templates of each 64-template tile with the sample index outermost: qt[tile][k][t]
// = q[tile 64 + t][k], so that a stage of K samples of a tile is one contiguous K x 64
// block. One block per (tile, 32 samples), through shared memory.
__global__ void k_template_tiles(const float *__restrict__ q, int m_pad, float *__restrict__ qt)
{
    __shared__ float sm[F_TPL][33];
    const int tile = blockIdx.y, k0 = blockIdx.x * 32;
    for (int i = threadIdx.x; i < F_TPL * 32; i += blockDim.x)
    {
        const int t = i >> 5, k = i & 31;
        sm[t][k] = q[(size_t)(tile * F_TPL + t) * m_pad + k0 + k];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < F_TPL * 32; i += blockDim.x)
    {
        const int k = i >> 6, t = i & 63;
        qt[((size_t)tile * m_pad + k0 + k) * F_TPL + t] = sm[t][k];
    }
}

cudaError_t launch_scan_fp32(const ScanArgs &a, cudaStream_t s)
{
    dim3 grid((a.W + F_WIN - 1) / F_WIN, (a.T + F_TPL - 1) / F_TPL);
    // m_pad is a multiple of 64, so of 32
    k_template_tiles<<<dim3((unsigned)(a.m_pad / 32), grid.y), 256, 0, s>>>(a.q, a.m_pad, a.qt);
    if (a.m_pad % 128 == 0)
    {
        cudaFuncSetAttribute(k_scan_fp32<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f_smem<128>());
        k_scan_fp32<128><<<grid, F_THREADS, f_smem<128>(), s>>>(a);
    }
    else
    {
        cudaFuncSetAttribute(k_scan_fp32<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f_smem<64>());
        k_scan_fp32<64><<<grid, F_THREADS, f_smem<64>(), s>>>(a);
    }
    return cudaGetLastError();
}

} // namespace tmb
