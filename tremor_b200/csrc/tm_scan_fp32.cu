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
    float(*qs)[F_TPL][F_K] = reinterpret_cast<float(*)[F_TPL][F_K]>(fsm + F_BUFS * F_XS_PAD);
    __shared__ TemplParam tps[F_TPL];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile_j = blockIdx.x * F_WIN;
    const int tile_t = blockIdx.y * F_TPL;
    if (tid < F_TPL)
        tps[tid] = a.tp[tile_t + tid];
    const uint32_t jmid = min(tile_j + F_WIN / 2, a.W - 1);
    const float shift = a.mean[jmid];
    const float *xg = a.x + a.w0 + tile_j;
    const float *qg = a.q + (size_t)tile_t * a.m_pad;

    auto load_stage = [&](int buf, int k0) {
        for (int i = tid; i < F_XS; i += F_THREADS)
            cp_async4(&xs[buf][xpos(i)], xg + k0 + i);
        for (int i = tid; i < F_TPL * F_K / 4; i += F_THREADS)
        {
            const int t = i / (F_K / 4), c = i % (F_K / 4);
            cp_async16(&qs[buf][t][c * 4], qg + (size_t)t * a.m_pad + k0 + c * 4);
        }
        cp_commit();
    };

    float acc[8][8];
#pragma unroll
    for (int w = 0; w < 8; w++)
#pragma unroll
        for (int t = 0; t < 8; t++)
            acc[w][t] = 0.0f;

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
        const float *qw = &qs[cur][8 * warp][0];
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
#pragma unroll
            for (int t = 0; t < 8; t++)
            {
                const float4 qv = *reinterpret_cast<const float4 *>(qw + t * F_K + kk);
#pragma unroll
                for (int w = 0; w < 8; w++)
                {
                    acc[w][t] = fmaf(xr[w + 0], qv.x, acc[w][t]);
                    acc[w][t] = fmaf(xr[w + 1], qv.y, acc[w][t]);
                    acc[w][t] = fmaf(xr[w + 2], qv.z, acc[w][t]);
                    acc[w][t] = fmaf(xr[w + 3], qv.w, acc[w][t]);
                }
            }
        }
    }

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

cudaError_t launch_scan_fp32(const ScanArgs &a, cudaStream_t s)
{
    dim3 grid((a.W + F_WIN - 1) / F_WIN, (a.T + F_TPL - 1) / F_TPL);
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
