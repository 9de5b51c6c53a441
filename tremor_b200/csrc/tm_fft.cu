// FFT contraction for few, long templates: FP64 overlap-save correlation of each template
// with the whole record, the same bounded epilogue as the contraction kernels, then the
// same exact re-scoring. TREMOR's FFT branch (fft_fallback.hpp:67-117, pieces and spectra
// fft_fallback.cpp:111-176) has this structure: FFT dot products with an error bound
// select windows that the exact kernel then verifies; MASS V3 (DMASS_V3.c:798-996) uses
// the same overlap-save pieces.
//
// Pieces: length kFftL = 32768 samples starting every kFftS = 16384 samples, so one set of
// spectra serves every template length m <= 16384: window j = p kFftS + o (0 <= o < kFftS)
// of piece p has its dot product at output o + m - 1 of the circular correlation, which
// does not wrap because o + m - 1 < kFftL. Each piece is shifted by s_p, its prefix block's
// centre rounded to float (exact in both precisions, so the epilogue's shift is exact).
//
// Error of an output (norm-wise, per piece; Higham, Accuracy and Stability of Numerical
// Algorithms, Thm 24.2, for FFTs of length L = 2^t in precision u with accurate twiddles:
// ||fl(FFT x) - FFT x||_2 <= kappa ||FFT x||_2, kappa ~ t (u + 4u sqrt 2)): with
// X = FFT(x - s_p), Y = FFT(reversed q), ||X||_2 = sqrt(L) ||x - s_p||_2,
// ||Y||_inf <= ||q||_1 <= sqrt(m) ||q||_2, ||X||_inf <= sqrt(L) ||x - s_p||_2,
//   ||fl(X) fl(Y) - X Y||_2 <= kappa sqrt(L) ||x - s_p|| ||q|| (sqrt m + sqrt L) (+ rounding),
//   ||fl(IFFT) - IFFT||: another kappa on ||X Y||_2 <= sqrt(L) ||x - s_p|| sqrt(m) ||q||,
// so every output's error is at most kappa ||x - s_p||_2 ||q||_2 (2 sqrt m + sqrt L). The
// library's FFT is not exactly radix-2 Cooley-Tukey; kappa is taken 10 times the theorem's.
#include "../../include/tremor_b200.h"
#include "tm_epilogue.cuh"
#include "tm_fft.cuh"

namespace tmb {

// 10 x log2(L) x (u + 4 u sqrt 2), u = 2^-53
constexpr double kFftKappa = 10.0 * 15.0 * (1.1102230246251565e-16 * (1.0 + 4.0 * 1.4142135623730951));

uint32_t fft_pieces(uint64_t n) { return (uint32_t)((n + kFftS - 1) / kFftS); }

// Pieces p0 .. p0 + count - 1 as FP64 (x - s_p, zero past n), their shifts and norms.
__global__ void __launch_bounds__(256) k_fft_gather(const float *__restrict__ clean, uint64_t n,
                                                    const double *__restrict__ centres, uint32_t p0,
                                                    double *__restrict__ pieces, double *__restrict__ shifts,
                                                    double *__restrict__ norms)
{
    __shared__ double part[8];
    const uint32_t p = p0 + blockIdx.x;
    const uint64_t start = (uint64_t)p * kFftS;
    const double s = (double)(float)centres[start >> kPrefixBlockLog];
    double *out = pieces + (size_t)blockIdx.x * kFftL;
    double sq = 0.0;
    for (int i = threadIdx.x; i < kFftL; i += blockDim.x)
    {
        const uint64_t g = start + (uint64_t)i;
        const double v = g < n ? (double)clean[g] - s : 0.0;
        out[i] = v;
        sq = fma(v, v, sq);
    }
    for (int off = 16; off > 0; off >>= 1)
        sq += __shfl_down_sync(0xffffffffu, sq, off);
    if ((threadIdx.x & 31) == 0)
        part[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++)
            t += part[w];
        shifts[p] = s;
        norms[p] = sqrt(t) * (1.0 + 1e-12); // rounding of the norm itself, generously
    }
}

// y = the template reversed and zero-padded to kFftL (FP64).
__global__ void k_fft_template(const float *__restrict__ q, int m, double *__restrict__ y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kFftL; i += gridDim.x * blockDim.x)
        y[i] = i < m ? (double)q[m - 1 - i] : 0.0;
}

// Z[p][k] = X[p][k] * Y[k] / L (the inverse FFT is unnormalised).
__global__ void k_fft_mul(const double2 *__restrict__ X, const double2 *__restrict__ Y, double2 *__restrict__ Z,
                          uint32_t count)
{
    const size_t total = (size_t)count * kFftH;
    const double inv = 1.0 / (double)kFftL;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
    {
        const double2 a = X[i], b = Y[i % kFftH];
        Z[i] = make_double2((a.x * b.x - a.y * b.y) * inv, (a.x * b.y + a.y * b.x) * inv);
    }
}


// One thread per window of the pieces: the distance and its bound as in the contraction
// kernels' epilogues (fast_distance_mixed), plus the FFT term 2 e_dot / sigma.
__global__ void __launch_bounds__(256) k_fft_epilogue(const FftEpiArgs f)
{
    const TemplParam p = f.p;
    const uint32_t lp = blockIdx.y;                    // piece within the batch
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t g = (uint64_t)(f.p0 + lp) * kFftS + o; // global window start
    const int lane = threadIdx.x & 31;
    const bool in_range = g >= f.w0 && g - f.w0 < p.wcount;
    const uint32_t jr = in_range ? (uint32_t)(g - f.w0) : 0u;
    bool ok = in_range && f.raw[g] != kMissing && f.run[g] < (uint16_t)min(p.m, 65535);
    float up = inf_f(), lo = inf_f();
    bool hit = false;
    if (ok)
    {
        WindowStats ws;
        if (window_prefix_stats(f.pv, f.pv.Q[g], f.pv.Q[g + (uint64_t)p.m], g, p.m, p.inv_m, ws) == 0)
        {
            const double dot = f.out[(size_t)lp * kFftL + o + (uint32_t)(p.m - 1)];
            const float shift = (float)f.shifts[f.p0 + lp];
            const float e_dot = (float)(kFftKappa * f.norms[f.p0 + lp] * f.e_fac * 1.01);
            float d, e;
            fast_distance_mixed(p, p.a1_main, (float)dot, ws.mu, ws.iv, shift, stats_error(ws, p.m, p.qs, p.s1), d,
                                e);
            e += 2.0f * e_dot * ws.iv * 1.01f;
            if (f.dbg_d != nullptr)
            {
                f.dbg_d[(size_t)f.t * f.W + jr] = d;
                f.dbg_e[(size_t)f.t * f.W + jr] = e;
            }
            up = d + e;
            lo = d - e;
            hit = lo <= p.thr_ed;
        }
        else
        {
            lo = -inf_f();
            hit = true;
        }
    }
    if (p.mode == TM_MODE_KNN)
    {
        // bucket minima: a warp's 32 windows lie in at most two buckets
        const uint32_t bucket = jr / kBucket;
        const unsigned act = __ballot_sync(0xffffffffu, in_range);
        if (act == 0u)
            return;
        const uint32_t b0 = __shfl_sync(0xffffffffu, bucket, __ffs(act) - 1);
        const unsigned same = __ballot_sync(0xffffffffu, in_range && bucket == b0);
        const unsigned other = act & ~same;
        const uint32_t ku = float_key(up), kl = float_key(lo);
        const uint32_t u0 = __reduce_min_sync(0xffffffffu, same & (1u << lane) ? ku : 0xffffffffu);
        const uint32_t l0 = __reduce_min_sync(0xffffffffu, same & (1u << lane) ? kl : 0xffffffffu);
        const uint32_t u1 = __reduce_min_sync(0xffffffffu, other & (1u << lane) ? ku : 0xffffffffu);
        const uint32_t l1 = __reduce_min_sync(0xffffffffu, other & (1u << lane) ? kl : 0xffffffffu);
        const uint32_t none = float_key(inf_f());
        if (lane == __ffs(act) - 1 && (u0 != none || l0 != none) && u0 != 0xffffffffu)
        {
            atomicMin(&f.bmin_u[(size_t)f.t * f.nb + b0], u0);
            atomicMin(&f.bmin_l[(size_t)f.t * f.nb + b0], l0);
        }
        if (other != 0u && lane == __ffs(other) - 1 && (u1 != none || l1 != none))
        {
            atomicMin(&f.bmin_u[(size_t)f.t * f.nb + bucket], u1);
            atomicMin(&f.bmin_l[(size_t)f.t * f.nb + bucket], l1);
        }
    }
    else
        emit_candidates(hit ? 1u : 0u, lane, f.t, jr, f.cand, f.cand_count, f.cand_cap);
}

cudaError_t launch_fft_gather(const float *clean, uint64_t n, const double *centres, uint32_t p0, uint32_t count,
                              double *pieces, double *shifts, double *norms, cudaStream_t s)
{
    if (count > 0)
        k_fft_gather<<<count, 256, 0, s>>>(clean, n, centres, p0, pieces, shifts, norms);
    return cudaGetLastError();
}

cudaError_t launch_fft_template(const float *q, int m, double *y, cudaStream_t s)
{
    k_fft_template<<<32, 256, 0, s>>>(q, m, y);
    return cudaGetLastError();
}

cudaError_t launch_fft_mul(const double2 *X, const double2 *Y, double2 *Z, uint32_t count, cudaStream_t s)
{
    if (count > 0)
        k_fft_mul<<<1184, 256, 0, s>>>(X, Y, Z, count);
    return cudaGetLastError();
}

cudaError_t launch_fft_epilogue(const FftEpiArgs &f, cudaStream_t s)
{
    if (f.count > 0)
        k_fft_epilogue<<<dim3(kFftS / 256, f.count), 256, 0, s>>>(f);
    return cudaGetLastError();
}

} // namespace tmb
