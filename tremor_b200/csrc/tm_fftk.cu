// In-tree FP64 FFT kernels of the FFT branch: the spectra of the record's pieces, the
// templates' spectra, and one fused kernel that correlates every template of a group with
// every piece and evaluates the distance bound, bucket minima and threshold candidates
// straight from shared memory. TREMOR's FFT branch (fft_fallback.hpp:67-117: per piece,
// the product with the template spectrum, an inverse real FFT, the dot product of each
// window and the distance filter with an error bound) has this structure; here neither the
// product spectrum nor the correlation leaves the SM.
//
// Two piece lengths, both with the step half the length (the window j = p S + o,
// 0 <= o < S, of piece p has its dot product at output o + m - 1 of the circular
// correlation, which does not wrap for m <= L - S + 1); each piece is shifted by s_p, the
// centre of the prefix block holding its start, rounded to float:
//   L = 16384, S = 8192  (kF2*): templates of up to 8192 samples;
//   L = 32768, S = 16384 (kF3*): templates of up to 16384 samples.
//
// Real transforms of length L go through complex ones of N = L / 2 points:
//   forward: z[n] = x[2n] + i x[2n+1], Z = FFT_N(z),
//            X[k] = (Z[k] + conj Z[N-k]) / 2 - i e^{-2 pi i k / L} (Z[k] - conj Z[N-k]) / 2;
//   inverse: for a Hermitian spectrum V (V[k] = X[k] Y[k]),
//            C[k] = (V[k] + conj V[N-k]) + i e^{2 pi i k / L} (V[k] - conj V[N-k]),
//            c = IFFT_N(C) (unnormalised), out[2n] = Re c[n], out[2n+1] = Im c[n],
//            and out / L is the circular correlation of x with the reversed template.
// Every complex transform is built from 8192-point ones, Stockham radix-16, 16, 16 then 2
// (Govindaraju et al., "High Performance Discrete Fourier Transforms on Graphics
// Processors", SC 2008): 512 threads, each holding 16 points in registers between a pass's
// shared-memory read and its write, so every pass works in place; the buffer is padded by
// one point per 16 so that the first pass's stride-16 writes hit distinct banks. The final
// radix-2 pass of an inverse is evaluated where its outputs are read (by the distance
// epilogue). For N = 16384 the forward transform splits z into its even and odd points
// (Z[k] = E[k] + W^k O[k], Z[k + 8192] = E[k] - W^k O[k], W = e^{-2 pi i / 16384}); the
// inverse splits C the other way (a[n] = C[n] + C[n + 8192] gives c[2k], b[n] = (C[n] -
// C[n + 8192]) e^{2 pi i n / 16384} gives c[2k + 1]), two 8192-point passes per piece.
//
// Twiddles: e^{2 pi i e / 32768} = R2[e >> 7] R1[e & 127] from tables of 128 and 256 entries
// computed on the host in extended precision and rounded (error <= 4u with u = 2^-53, the
// product included); a pass's powers w^r (r = 1..15) by repeated multiplication (error
// <= 7 r u <= 105u). Error of an output (Higham, Accuracy and Stability of Numerical
// Algorithms, Thm 24.2, ||fl(FFT x) - FFT x||_2 <= t eta / (1 - t eta) ||FFT x||_2,
// eta = mu + gamma_4 (sqrt 2 + mu), mu the twiddle error): with mu = 105u, t = log2 L + 2
// (the complex stages plus the real-transform packing and the even/odd split) and a factor
// 10 for the radix-16 and packing arithmetic, kappa = 10 t 111u. With X = FFT(x - s_p),
// Y = FFT(reversed q), ||X||_2 = sqrt(L) ||x - s_p||_2, ||Y||_inf <= ||q||_1 <= sqrt(m)
// ||q||_2: ||fl(X) fl(Y) - X Y||_2 <= kappa sqrt(L) ||x - s_p|| ||q|| (sqrt m + sqrt L)
// (+ rounding), and the inverse adds kappa ||X Y||_2 <= kappa sqrt(L) ||x - s_p|| sqrt(m)
// ||q||, so every correlation output is within kappa ||x - s_p||_2 ||q||_2 (2 sqrt m +
// sqrt L) of the exact one.
#include <cmath>

#include "../../include/tremor_b200.h"
#include "tm_epilogue.cuh"
#include "tm_fft.cuh"

namespace tmb {

constexpr int kF2T = 512;                        // threads per block
constexpr int kFPts = 8192;                      // points of the in-shared-memory transforms
constexpr int kF2Buf = kFPts + kFPts / 16 + 16;  // padded complex entries of the work buffer
constexpr int kFRoots = 384;                     // twiddle table entries (R1 then R2)
constexpr double kF2Kappa = 10.0 * 16.0 * 111.0 * 1.1102230246251565e-16;
constexpr double kF3Kappa = 10.0 * 17.0 * 111.0 * 1.1102230246251565e-16;
constexpr size_t kF2Smem = sizeof(double2) * (size_t)(kF2Buf + kFRoots);

__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }
// a * (s i): s = +1 or -1
template <int S> __device__ __forceinline__ double2 mul_si(double2 a)
{
    return S > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// Position of R1[a] in shared memory: the low three bits XOR-ed with bits 3-5, so that the
// lookups of a quarter warp at strides 1, 2, 4 or 8 (the passes' and epilogue's patterns)
// fall in distinct banks.
__device__ __forceinline__ int r1_slot(int a) { return a ^ ((a >> 3) & 7); }

// e^{S 2 pi i e / 32768}, 0 <= e < 32768, from the shared tables R (R1 then R2).
template <int S> __device__ __forceinline__ double2 root(const double2 *R, int e)
{
    const double2 w = cmul(R[128 + (e >> 7)], R[r1_slot(e & 127)]);
    return S > 0 ? w : conj2(w);
}

// 4-point DFT with e^{S 2 pi i / 4} = S i, in place on x0..x3.
template <int S> __device__ __forceinline__ void dft4(double2 &x0, double2 &x1, double2 &x2, double2 &x3)
{
    const double2 a = cadd(x0, x2), b = csub(x0, x2), c = cadd(x1, x3), d = mul_si<S>(csub(x1, x3));
    x0 = cadd(a, c);
    x2 = csub(a, c);
    x1 = cadd(b, d);
    x3 = csub(b, d);
}

// 16-point DFT in natural order, as 4 x 4: t[b][c] = DFT4_a(v[4a + b])[c], times
// W16^{bc}, then X[c + 4d] = DFT4_b(t[b][c])[d].
template <int S> __device__ __forceinline__ void dft16(double2 (&v)[16])
{
    constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173, h = 0.70710678118654752440;
#pragma unroll
    for (int b = 0; b < 4; b++)
        dft4<S>(v[b], v[4 + b], v[8 + b], v[12 + b]); // v[4c + b] now holds t[b][c]
    // twiddles W16^{bc} (b, c = 1..3): exponents 1, 2, 3, 2, 4, 6, 3, 6, 9
    const double2 w1 = make_double2(c1, S * s1), w2 = make_double2(h, S * h), w3 = make_double2(s1, S * c1);
    const double2 w6 = make_double2(-h, S * h), w9 = make_double2(-c1, -S * s1);
    v[4 + 1] = cmul(v[4 + 1], w1);
    v[8 + 1] = cmul(v[8 + 1], w2);
    v[12 + 1] = cmul(v[12 + 1], w3);
    v[4 + 2] = cmul(v[4 + 2], w2);
    v[8 + 2] = mul_si<S>(v[8 + 2]); // W16^4 = S i
    v[12 + 2] = cmul(v[12 + 2], w6);
    v[4 + 3] = cmul(v[4 + 3], w3);
    v[8 + 3] = cmul(v[8 + 3], w6);
    v[12 + 3] = cmul(v[12 + 3], w9);
#pragma unroll
    for (int c = 0; c < 4; c++)
        dft4<S>(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]); // X[c + 4d] in v[4c + d]
    // natural order: X[c + 4d] from v[4c + d] (a 4 x 4 transpose of registers)
#pragma unroll
    for (int c = 0; c < 4; c++)
#pragma unroll
        for (int d = c + 1; d < 4; d++)
        {
            const double2 t = v[4 * c + d];
            v[4 * c + d] = v[4 * d + c];
            v[4 * d + c] = t;
        }
}

// One Stockham radix-16 pass over the padded buffer (N = 8192, 512 threads, in place: every
// thread reads its 16 points, the block synchronises, then every thread writes).
template <int S> __device__ __forceinline__ void pass16(double2 *buf, const double2 *R, int Ns)
{
    const int j = threadIdx.x;
    double2 v[16];
#pragma unroll
    for (int r = 0; r < 16; r++)
        v[r] = buf[pidx(j + 512 * r)];
    __syncthreads();
    const int k = j & (Ns - 1);
    if (Ns > 1)
    {
        const double2 w1 = root<S>(R, k * (2048 / Ns)); // W^k, W = e^{S 2 pi i / (16 Ns)}
        double2 w = w1;
#pragma unroll
        for (int r = 1; r < 16; r++)
        {
            v[r] = cmul(v[r], w);
            if (r < 15)
                w = cmul(w, w1);
        }
    }
    dft16<S>(v);
    const int d0 = (j - k) * 16 + k;
#pragma unroll
    for (int r = 0; r < 16; r++)
        buf[pidx(d0 + r * Ns)] = v[r];
    __syncthreads();
}

// The three radix-16 passes of an 8192-point transform; the radix-2 pass is left to the
// caller (final_out, or the forward kernel's explicit pass).
template <int S> __device__ __forceinline__ void fft8192_r16(double2 *buf, const double2 *R)
{
    pass16<S>(buf, R, 1);
    pass16<S>(buf, R, 16);
    pass16<S>(buf, R, 256);
}

// Output i (0 <= i < 8192) of the final radix-2 pass: c[i] = a + w b, c[i + 4096] = a - w b
// with a = buf[i mod 4096], b = buf[i mod 4096 + 4096], w = e^{S 2 pi i (i mod 4096) / 8192}.
template <int S> __device__ __forceinline__ double2 final_out(const double2 *buf, const double2 *R, int i)
{
    const int i0 = i & 4095;
    const double2 a = buf[pidx(i0)], b = cmul(buf[pidx(i0 + 4096)], root<S>(R, 4 * i0));
    return i < 4096 ? cadd(a, b) : csub(a, b);
}

__device__ __forceinline__ void load_roots(double2 *R, const double2 *roots)
{
    for (int i = threadIdx.x; i < kFRoots; i += blockDim.x)
        R[i < 128 ? r1_slot(i) : i] = roots[i];
}

// What the epilogue reads from global memory for one window: its prefix sums at the start
// and the end, its first sample and its constant run. The epilogues load these for a few
// windows at once before evaluating any of them, so that the loads overlap (with one block
// of 512 threads per SM there are too few warps to hide one load's latency at a time).
struct WinIn
{
    double2 qa, qb;
    float raw;
    uint32_t run;
};

__device__ __forceinline__ WinIn load_window(const Fft2Args &a, int m, bool in_range, uint64_t g)
{
    WinIn w;
    if (in_range)
    {
        w.qa = a.pv.Q[g];
        w.qb = a.pv.Q[g + (uint64_t)m];
        w.raw = a.raw[g];
        w.run = a.run[g];
    }
    else
    {
        w.qa = w.qb = make_double2(0.0, 0.0);
        w.raw = kMissing;
        w.run = 0;
    }
    return w;
}

// A window's statistics as the epilogue uses them, for one template length: x = mean,
// y = 1 / std, z and w the two factors of its error term (WindowStats::rel_sd, e_mu);
// y == 0: the window is not searched (outside the range, first sample missing, constant);
// y < 0: its statistics are not trusted (it is re-scored exactly whatever its distance).
// They do not depend on the template: the epilogues fold them (fold_window) and keep them in
// the block's slice of a global scratch (L2-resident) for the next template of the same
// length in the same piece.
// Single-block, well-conditioned windows take the fast path (prefix_stats_fast), the others
// the full bound.
__device__ __forceinline__ float4 window_stats4(const Fft2Args &a, int m, double inv_m, bool in_range, uint64_t g,
                                                const WinIn &w)
{
    if (!(in_range && w.raw != kMissing && w.run < (uint32_t)min(m, 65535)))
        return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const uint64_t b1 = g >> kPrefixBlockLog;
    if (((g + (uint64_t)m) >> kPrefixBlockLog) == b1)
    {
        float mu, iv, emu;
        if (prefix_stats_fast(w.qa, w.qb, inv_m, (float)inv_m * (1.0f + 1.1920929e-07f), (float)a.pv.C[b1],
                              block_bounds(a.pv.T[b1].y), mu, iv, emu))
            return make_float4(mu, iv, kFastRelSd, emu);
    }
    WindowStats ws;
    if (window_prefix_stats(a.pv, w.qa, w.qb, g, m, inv_m, ws) != 0)
        return make_float4(0.0f, -1.0f, 0.0f, 0.0f);
    return make_float4(ws.mu, ws.iv, ws.rel_sd, ws.e_mu);
}

// The folded statistics of a window for the templates of one length in one piece (what the
// block's cache holds): x = mu - shift, y = 1 / std as in window_stats4 (0: not searched;
// < 0: statistics not trusted), z = every term of the distance bound that does not depend
// on the dot product's distance: fast_distance_mixed's bound without its a3 max(d, 0) term,
// with the largest coefficients c0 = (a1, a2, a5, a6), c1 = (qs, |s1|) of the launch's
// templates of this length (so it bounds each of them), plus the transform's error
// 2 e_dot / std.
__device__ __forceinline__ float4 fold_window(const float4 &st, const float4 &c0, const float4 &c1, int m, float shift,
                                              float e_dot)
{
    if (!(st.y > 0.0f))
        return make_float4(0.0f, st.y, 0.0f, 0.0f);
    const float mu = st.x, iv = st.y, ms = mu - shift;
    const float r = ms * iv, r0 = mu * iv;
    WindowStats ws;
    ws.mu = mu;
    ws.iv = iv;
    ws.rel_sd = st.z;
    ws.e_mu = st.w;
    const float ew = c0.x * sqrtf(1.0f + r * r) + c0.y + c0.z * r0 * r0 + c0.w * (fabsf(mu) + fabsf(shift)) * iv +
                     stats_error(ws, m, c1.x, c1.y) + 2.0f * e_dot * iv * 1.01f;
    return make_float4(ms, iv, ew, 0.0f);
}

// The per-template epilogue of window jr (relative to w0) with folded statistics st and dot
// product dot: d as fast_distance_mixed, up = d + e and lo = d - e (+inf for windows not
// searched; lo = -inf when the statistics are not trusted), hit = lo <= the threshold
// distance.
__device__ __forceinline__ void corr_eval(const Fft2Args &a, const TemplParam &P, int t, uint32_t jr, const float4 &st,
                                          double dot, float &up, float &lo, bool &hit)
{
    up = inf_f();
    lo = inf_f();
    hit = false;
    if (st.y == 0.0f)
        return;
    if (st.y > 0.0f)
    {
        const float cross = ((float)dot - st.x * P.s1) * st.y;
        const float d = P.c_lin - 2.0f * cross;
        const float e = st.z + P.a3 * fmaxf(d, 0.0f);
        if (a.dbg_d != nullptr)
        {
            a.dbg_d[(size_t)t * a.W + jr] = d;
            a.dbg_e[(size_t)t * a.W + jr] = e;
        }
        up = d + e;
        lo = d - e;
        hit = lo <= P.thr_ed;
    }
    else
    {
        lo = -inf_f();
        hit = true;
    }
}

// kNN bucket minima of a group of J windows per lane (windows jr[j] relative to w0, those
// with inr[j] in the template's range) whose warp-wide span is under a bucket, so they lie in
// at most two buckets B and B + 1: per-lane minima first, then one warp reduction per bucket
// and key, and one atomic per bucket and key (skipped for buckets with no searched window,
// whose minima stay at +inf's key). Every lane of the warp must call it.
template <int J>
__device__ __forceinline__ void bucket_minima(const Fft2Args &a, int t, int lane, const bool (&inr)[J],
                                              const uint32_t (&jr)[J], const float (&up)[J], const float (&lo)[J])
{
    uint32_t bmin = 0xffffffffu;
#pragma unroll
    for (int j = 0; j < J; j++)
        if (inr[j])
            bmin = min(bmin, jr[j] / (uint32_t)kBucket);
    const uint32_t B = __reduce_min_sync(0xffffffffu, bmin);
    if (B == 0xffffffffu)
        return; // no window of the warp in the range
    uint32_t uA = 0xffffffffu, lA = 0xffffffffu, uB = 0xffffffffu, lB = 0xffffffffu;
#pragma unroll
    for (int j = 0; j < J; j++)
    {
        if (!inr[j])
            continue;
        const uint32_t ku = float_key(up[j]), kl = float_key(lo[j]);
        if (jr[j] / (uint32_t)kBucket == B)
        {
            uA = min(uA, ku);
            lA = min(lA, kl);
        }
        else
        {
            uB = min(uB, ku);
            lB = min(lB, kl);
        }
    }
    uA = __reduce_min_sync(0xffffffffu, uA);
    lA = __reduce_min_sync(0xffffffffu, lA);
    uB = __reduce_min_sync(0xffffffffu, uB);
    lB = __reduce_min_sync(0xffffffffu, lB);
    const uint32_t none = float_key(inf_f());
    if (lane == 0)
    {
        if (uA != 0xffffffffu && (uA != none || lA != none))
        {
            atomicMin(&a.bmin_u[(size_t)t * a.nb + B], uA);
            atomicMin(&a.bmin_l[(size_t)t * a.nb + B], lA);
        }
        if (uB != 0xffffffffu && (uB != none || lB != none))
        {
            atomicMin(&a.bmin_u[(size_t)t * a.nb + B + 1], uB);
            atomicMin(&a.bmin_l[(size_t)t * a.nb + B + 1], lB);
        }
    }
}

// Threshold candidates of one window per lane: one ballot, one atomic per warp with hits.
// Entries past the capacity are counted, not written. Every lane of the warp must call it.
__device__ __forceinline__ void emit_hits(const Fft2Args &a, int t, int lane, bool hit, uint32_t jr)
{
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (b == 0u)
        return;
    const int leader = __ffs(b) - 1;
    uint32_t base = 0;
    if (lane == leader)
        base = atomicAdd(a.cand_count, (uint32_t)__popc(b));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (hit)
    {
        const uint32_t pos = base + (uint32_t)__popc(b & ((1u << lane) - 1u));
        if (pos < a.cand_cap)
            a.cand[pos] = Candidate{(uint32_t)t, jr};
    }
}

// Forward real FFT of one piece of the record (blockIdx.x < pieces) or one template row
// (templates: reversed and zero-padded to kF2L), into out[blockIdx.x * kF2H ..].
__global__ void __launch_bounds__(kF2T, 1) k_fft2_forward(const float *__restrict__ clean, uint64_t n,
                                                         const double *__restrict__ centres, uint32_t p0,
                                                         const float *__restrict__ q, const TemplParam *__restrict__ tp,
                                                         const int *__restrict__ rows, const double2 *__restrict__ roots,
                                                         double2 *__restrict__ out, double *__restrict__ shifts,
                                                         double *__restrict__ norms)
{
    extern __shared__ double2 sm2[];
    double2 *buf = sm2, *R = sm2 + kF2Buf;
    __shared__ double part[kF2T / 32];
    load_roots(R, roots);
    const bool templ = q != nullptr;
    double s = 0.0, sq = 0.0;
    uint64_t start = 0;
    const float *qt = nullptr;
    int m = 0;
    if (templ)
    {
        const TemplParam &p = tp[rows[blockIdx.x]];
        qt = q + p.q_offset;
        m = p.m;
    }
    else
    {
        start = (uint64_t)(p0 + blockIdx.x) * kF2S;
        s = (double)(float)centres[start >> kPrefixBlockLog];
    }
    for (int i = threadIdx.x; i < kF2N; i += kF2T)
    {
        double a, b;
        if (templ)
        {
            const int i0 = 2 * i, i1 = 2 * i + 1; // y[i] = q[m - 1 - i]
            a = i0 < m ? (double)qt[m - 1 - i0] : 0.0;
            b = i1 < m ? (double)qt[m - 1 - i1] : 0.0;
        }
        else
        {
            const uint64_t g = start + 2 * (uint64_t)i;
            a = g < n ? (double)clean[g] - s : 0.0;
            b = g + 1 < n ? (double)clean[g + 1] - s : 0.0;
            sq = fma(a, a, sq);
            sq = fma(b, b, sq);
        }
        buf[pidx(i)] = make_double2(a, b);
    }
    __syncthreads();
    fft8192_r16<-1>(buf, R);
    // the radix-2 pass, in place (each thread owns the pairs (i, i + 4096) it touches)
    for (int i = threadIdx.x; i < 4096; i += kF2T)
    {
        const double2 a = buf[pidx(i)], b = cmul(buf[pidx(i + 4096)], root<-1>(R, 4 * i));
        buf[pidx(i)] = cadd(a, b);
        buf[pidx(i + 4096)] = csub(a, b);
    }
    __syncthreads();
    double2 *o = out + (size_t)blockIdx.x * kF2H;
    for (int k = threadIdx.x; k <= kF2N / 2; k += kF2T)
    {
        // X[k] and X[N - k] from Z[k] and Z[N - k] (Z[N] = Z[0])
        const double2 A = buf[pidx(k)], Bc = conj2(buf[pidx(k == 0 ? 0 : kF2N - k)]);
        const double2 E = make_double2(0.5 * (A.x + Bc.x), 0.5 * (A.y + Bc.y));
        const double2 D = csub(A, Bc);
        const double2 O = make_double2(0.5 * D.y, -0.5 * D.x); // -i (A - B) / 2
        const double2 w = root<-1>(R, 2 * k);                   // e^{-2 pi i k / L}
        o[k] = cadd(E, cmul(O, w));
        if (k == 0)
            o[kF2N] = csub(E, O); // twiddle e^{-i pi} = -1
        else if (k < kF2N / 2)
        {
            const double2 A2 = conj2(Bc), B2c = conj2(A); // Z[N - k], conj Z[k]
            const double2 E2 = make_double2(0.5 * (A2.x + B2c.x), 0.5 * (A2.y + B2c.y));
            const double2 D2 = csub(A2, B2c);
            const double2 O2 = make_double2(0.5 * D2.y, -0.5 * D2.x);
            o[kF2N - k] = csub(E2, cmul(O2, conj2(w))); // e^{-2 pi i (N - k) / L} = -e^{2 pi i k / L}
        }
    }
    if (!templ)
    {
        for (int off = 16; off > 0; off >>= 1)
            sq += __shfl_down_sync(0xffffffffu, sq, off);
        if ((threadIdx.x & 31) == 0)
            part[threadIdx.x >> 5] = sq;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double t = 0.0;
            for (int w = 0; w < kF2T / 32; w++)
                t += part[w];
            shifts[p0 + blockIdx.x] = s;
            norms[p0 + blockIdx.x] = sqrt(t) * (1.0 + 1e-12); // rounding of the norm itself, generously
        }
    }
}

// The fused correlation: persistent blocks over pieces; per piece, every template of the
// launch: C from X[p] Y[t] (the product and the real-transform packing in one step), the
// radix-16 passes, then one thread per window: its dot product from the final radix-2
// pass, the distance and bound as the contraction kernels' epilogues (fast_distance_mixed
// with prefix-sum statistics) plus the FFT's own error, then kNN bucket minima or threshold
// candidates.
__global__ void __launch_bounds__(kF2T, 1) k_fft2_corr(const Fft2Args a)
{
    extern __shared__ double2 sm2[];
    __shared__ TemplParam sP;
    double2 *buf = sm2, *R = sm2 + kF2Buf;
    load_roots(R, a.roots);
    const int lane = threadIdx.x & 31;
    const double inv_l = 1.0 / (double)kF2L;
    float4 *cache = a.stats + (size_t)blockIdx.x * kFftCache; // this block's statistics cache
    for (uint32_t pi = blockIdx.x; pi < a.p_count; pi += gridDim.x)
    {
        int cached_m = -1; // the length whose statistics of this piece the cache holds
        const uint32_t p = a.p_first + pi;
        const double2 *X = a.X + (size_t)p * kF2H;
        const float shift = (float)a.shifts[p];
        const double norm = a.norms[p];
        for (int ti = 0; ti < a.nrows; ti++)
        {
            const int t = a.rows[ti];
            const uint64_t piece_w = (uint64_t)p * kF2S;
            // windows of this piece in the template's range [w0, w0 + wcount)
            const uint64_t wcount = a.tp[t].wcount;
            if (piece_w + kF2S <= a.w0 || piece_w >= a.w0 + wcount)
                continue;
            const double2 *Y = a.Y + (size_t)ti * kF2H;
            __syncthreads(); // the previous template's epilogue has read buf and sP
            if (threadIdx.x == 0)
                sP = a.tp[t]; // the template's constants, read by every thread from shared memory
            const TemplParam &P = sP;
            // work items k = thread + 512 i (0 <= k <= N / 2), two at a time: their spectrum
            // loads first, then the products
            for (int i0 = 0; i0 < 10; i0 += 2)
            {
                double2 xk[2], xn[2], yk[2], yn[2];
#pragma unroll
                for (int j = 0; j < 2; j++)
                {
                    const int k = (int)threadIdx.x + kF2T * (i0 + j);
                    if (k <= kF2N / 2)
                    {
                        xk[j] = X[k];
                        xn[j] = X[kF2N - k];
                        yk[j] = Y[k];
                        yn[j] = Y[kF2N - k];
                    }
                }
#pragma unroll
                for (int j = 0; j < 2; j++)
                {
                    const int k = (int)threadIdx.x + kF2T * (i0 + j), kn = kF2N - k;
                    if (k > kF2N / 2)
                        continue;
                    const double2 Vk = cmul(xk[j], yk[j]), Vn = cmul(xn[j], yn[j]);
                    const double2 w = root<1>(R, 2 * k); // e^{2 pi i k / L}
                    // C[k] = E + i O with E = Vk + conj Vn, O = w (Vk - conj Vn); C[N - k] = conj E + i conj O
                    const double2 E = cadd(Vk, conj2(Vn));
                    const double2 O = cmul(csub(Vk, conj2(Vn)), w);
                    if (k == 0)
                        buf[pidx(0)] = cadd(E, mul_si<1>(O)); // C[0] (Vn = V[N], the Nyquist bin)
                    else
                    {
                        buf[pidx(k)] = cadd(E, mul_si<1>(O));
                        if (k < kF2N / 2)
                            buf[pidx(kn)] = cadd(conj2(E), mul_si<1>(conj2(O)));
                    }
                }
            }
            __syncthreads();
            fft8192_r16<1>(buf, R);
            // epilogue: work item u = it * 512 + thread takes output i = (base >> 1) + u of the
            // final pass (base = m - 1), whose real and imaginary parts are the dot products of
            // windows o = 2 u - odd and 2 u - odd + 1 (odd = base & 1; with odd base, item 0
            // has only window 0 and item 4096 only window 8191). Window o is in the template's
            // range when o_lo <= o < o_hi; jr = rel + o is its index relative to w0.
            const int base = P.m - 1, odd = base & 1, nitems = kF2S / 2 + odd;
            const int64_t rel = (int64_t)piece_w - (int64_t)a.w0;
            const int o_lo = (int)(rel < 0 ? -rel : 0);
            const int o_hi = (int)((int64_t)P.wcount - rel < (int64_t)kF2S ? (int64_t)P.wcount - rel : (int64_t)kF2S);
            const double sm_ = sqrt((double)P.m);
            const float e_dot = (float)(kF2Kappa * norm * sm_ * (2.0 * sm_ + sqrt((double)kF2L)) * 1.01);
            // the windows' folded statistics: computed for the first template of a length in
            // this piece, then read back from the block's cache (each thread reads what it wrote)
            const bool cached = P.m == cached_m;
            const float4 c0 = a.gmax[2 * t], c1 = a.gmax[2 * t + 1];
            for (int it0 = 0; it0 < 10; it0 += 2)
            {
                if (it0 * kF2T + (int)(threadIdx.x & ~31u) >= nitems)
                    continue; // no item of this warp (uniform across the warp)
                float4 st[4];
                bool inr[4], hit[4];
                uint32_t jr[4];
                float up[4], lo[4];
#pragma unroll
                for (int j = 0; j < 4; j++)
                {
                    const int u = (it0 + (j >> 1)) * kF2T + (int)threadIdx.x;
                    const int o = 2 * u - odd + (j & 1);
                    inr[j] = u < nitems && o >= o_lo && o < o_hi;
                    jr[j] = (uint32_t)rel + (uint32_t)o;
                }
                if (cached)
                {
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        st[j] = inr[j] ? cache[2 * ((it0 + (j >> 1)) * kF2T + (int)threadIdx.x) + (j & 1)]
                                       : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                }
                else
                {
                    WinIn w[4];
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        w[j] = load_window(a, P.m, inr[j], (uint64_t)((int64_t)a.w0 + (int64_t)jr[j]));
#pragma unroll
                    for (int j = 0; j < 4; j++)
                    {
                        st[j] = fold_window(window_stats4(a, P.m, P.inv_m, inr[j],
                                                          (uint64_t)((int64_t)a.w0 + (int64_t)jr[j]), w[j]),
                                            c0, c1, P.m, shift, e_dot);
                        if (inr[j])
                            cache[2 * ((it0 + (j >> 1)) * kF2T + (int)threadIdx.x) + (j & 1)] = st[j];
                    }
                }
#pragma unroll
                for (int j = 0; j < 4; j += 2)
                {
                    const int u = (it0 + (j >> 1)) * kF2T + (int)threadIdx.x;
                    double2 c = make_double2(0.0, 0.0);
                    if (inr[j] || inr[j + 1])
                        c = final_out<1>(buf, R, (base >> 1) + u);
                    corr_eval(a, P, t, jr[j], st[j], c.x * inv_l, up[j], lo[j], hit[j]);
                    corr_eval(a, P, t, jr[j + 1], st[j + 1], c.y * inv_l, up[j + 1], lo[j + 1], hit[j + 1]);
                }
                if (P.mode == TM_MODE_KNN)
                    bucket_minima<4>(a, t, lane, inr, jr, up, lo); // the group spans 512 x 2 + 64 windows
                else
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        emit_hits(a, t, lane, hit[j], jr[j]);
            }
            cached_m = P.m;
        }
    }
}

// Forward real FFT of length kF3L of pieces (item i: piece p0 + i) or template rows (item i:
// rows[i], reversed and zero-padded), into out[item * kF3H ..]: persistent blocks, the
// even-point transform E parked in the block's slice of `scratch` (kFPts points) while the
// odd-point one O stays in shared memory, then the two combined and unpacked.
__global__ void __launch_bounds__(kF2T, 1) k_fft3_forward(const float *__restrict__ clean, uint64_t n,
                                                         const double *__restrict__ centres, uint32_t p0,
                                                         uint32_t count, const float *__restrict__ q,
                                                         const TemplParam *__restrict__ tp, const int *__restrict__ rows,
                                                         const double2 *__restrict__ roots, double2 *__restrict__ out,
                                                         double *__restrict__ shifts, double *__restrict__ norms,
                                                         double2 *__restrict__ scratch)
{
    extern __shared__ double2 sm2[];
    double2 *buf = sm2, *R = sm2 + kF2Buf;
    __shared__ double part[kF2T / 32];
    load_roots(R, roots);
    double2 *Es = scratch + (size_t)blockIdx.x * kFPts;
    const bool templ = q != nullptr;
    for (uint32_t item = blockIdx.x; item < count; item += gridDim.x)
    {
        double s = 0.0, sq = 0.0;
        uint64_t start = 0;
        const float *qt = nullptr;
        int m = 0;
        if (templ)
        {
            const TemplParam &p = tp[rows[item]];
            qt = q + p.q_offset;
            m = p.m;
        }
        else
        {
            start = (uint64_t)(p0 + item) * kF3S;
            s = (double)(float)centres[start >> kPrefixBlockLog];
        }
        for (int half = 0; half < 2; half++)
        {
            __syncthreads(); // buf and Es are free (the previous half's or item's readers are done)
            for (int i = threadIdx.x; i < kFPts; i += kF2T)
            {
                // point 2i + half of z: samples 4i + 2 half and 4i + 2 half + 1
                const uint64_t t0 = 4 * (uint64_t)i + 2 * (uint64_t)half;
                double va, vb;
                if (templ)
                {
                    va = t0 < (uint64_t)m ? (double)qt[m - 1 - (int)t0] : 0.0;
                    vb = t0 + 1 < (uint64_t)m ? (double)qt[m - 2 - (int)t0] : 0.0;
                }
                else
                {
                    const uint64_t g = start + t0;
                    va = g < n ? (double)clean[g] - s : 0.0;
                    vb = g + 1 < n ? (double)clean[g + 1] - s : 0.0;
                    sq = fma(va, va, sq);
                    sq = fma(vb, vb, sq);
                }
                buf[pidx(i)] = make_double2(va, vb);
            }
            __syncthreads();
            fft8192_r16<-1>(buf, R);
            for (int i = threadIdx.x; i < 4096; i += kF2T)
            {
                const double2 x0 = buf[pidx(i)], x1 = cmul(buf[pidx(i + 4096)], root<-1>(R, 4 * i));
                buf[pidx(i)] = cadd(x0, x1);
                buf[pidx(i + 4096)] = csub(x0, x1);
            }
            __syncthreads();
            if (half == 0)
                for (int k = threadIdx.x; k < kFPts; k += kF2T)
                    Es[k] = buf[pidx(k)];
        }
        __syncthreads(); // Es written, buf holds O
        // Z[k] = E[k] + W^k O[k] (k < 8192), Z[k + 8192] = E[k] - W^k O[k], W^k = e^{-2 pi i k / 16384}
        auto Z = [&](int k) -> double2 {
            const int k0 = k & (kFPts - 1);
            const double2 wo = cmul(buf[pidx(k0)], root<-1>(R, 2 * k0));
            return k < kFPts ? cadd(Es[k0], wo) : csub(Es[k0], wo);
        };
        constexpr int N = kF3N;
        double2 *o = out + (size_t)item * kF3H;
        for (int k = threadIdx.x; k <= N / 2; k += kF2T)
        {
            const double2 A = Z(k), Bc = conj2(Z(k == 0 ? 0 : N - k));
            const double2 E = make_double2(0.5 * (A.x + Bc.x), 0.5 * (A.y + Bc.y));
            const double2 D = csub(A, Bc);
            const double2 O = make_double2(0.5 * D.y, -0.5 * D.x);
            const double2 w = root<-1>(R, k); // e^{-2 pi i k / 32768}
            o[k] = cadd(E, cmul(O, w));
            if (k == 0)
                o[N] = csub(E, O);
            else if (k < N / 2)
            {
                const double2 A2 = conj2(Bc), B2c = conj2(A);
                const double2 E2 = make_double2(0.5 * (A2.x + B2c.x), 0.5 * (A2.y + B2c.y));
                const double2 D2 = csub(A2, B2c);
                const double2 O2 = make_double2(0.5 * D2.y, -0.5 * D2.x);
                o[N - k] = csub(E2, cmul(O2, conj2(w)));
            }
        }
        if (!templ)
        {
            for (int off = 16; off > 0; off >>= 1)
                sq += __shfl_down_sync(0xffffffffu, sq, off);
            if ((threadIdx.x & 31) == 0)
                part[threadIdx.x >> 5] = sq;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                double tot = 0.0;
                for (int w = 0; w < kF2T / 32; w++)
                    tot += part[w];
                shifts[p0 + item] = s;
                norms[p0 + item] = sqrt(tot) * (1.0 + 1e-12);
            }
        }
    }
}

// The fused correlation for pieces of kF3L samples (templates of up to kF3S samples): per
// piece and template, two halves h = 0, 1: the product with the template spectrum, the
// real-transform packing and the even/odd split in one step (h = 0: a[n] = C[n] + C[n + 8192];
// h = 1: b[n] = (C[n] - C[n + 8192]) e^{2 pi i n / 16384}), the radix-16 passes, then the
// windows whose output index has c index parity h (out[n0] with (n0 >> 1) & 1 == h, two of
// every four consecutive windows), each from the final radix-2 pass.
__global__ void __launch_bounds__(kF2T, 1) k_fft3_corr(const Fft2Args a)
{
    extern __shared__ double2 sm2[];
    __shared__ TemplParam sP;
    double2 *buf = sm2, *R = sm2 + kF2Buf;
    load_roots(R, a.roots);
    const int lane = threadIdx.x & 31;
    const double inv_l = 1.0 / (double)kF3L;
    constexpr int N = kF3N;
    float4 *cache = a.stats + (size_t)blockIdx.x * kFftCache; // this block's statistics cache
    for (uint32_t pi = blockIdx.x; pi < a.p_count; pi += gridDim.x)
    {
        int cached_m = -1; // the length whose statistics of this piece the cache holds
        const uint32_t p = a.p_first + pi;
        const double2 *X = a.X + (size_t)p * kF3H;
        const float shift = (float)a.shifts[p];
        const double norm = a.norms[p];
        for (int ti = 0; ti < a.nrows; ti++)
        {
            const int t = a.rows[ti];
            const uint64_t piece_w = (uint64_t)p * kF3S;
            const uint64_t wcount = a.tp[t].wcount;
            if (piece_w + kF3S <= a.w0 || piece_w >= a.w0 + wcount)
                continue;
            const double2 *Y = a.Y + (size_t)ti * kF3H;
            __syncthreads(); // the previous template's epilogue has read sP
            if (threadIdx.x == 0)
                sP = a.tp[t]; // the template's constants, read by every thread from shared memory
            __syncthreads();
            const TemplParam &P = sP;
            const double sm_ = sqrt((double)P.m);
            const float e_dot = (float)(kF3Kappa * norm * sm_ * (2.0 * sm_ + sqrt((double)kF3L)) * 1.01);
            const int base = P.m - 1;
            const bool cached = P.m == cached_m; // (each thread reads back only what it wrote)
            const float4 c0 = a.gmax[2 * t], c1 = a.gmax[2 * t + 1];
            const int64_t rel = (int64_t)piece_w - (int64_t)a.w0;
            const int o_lo = (int)(rel < 0 ? -rel : 0);
            const int o_hi = (int)((int64_t)P.wcount - rel < (int64_t)kF3S ? (int64_t)P.wcount - rel : (int64_t)kF3S);
            for (int h = 0; h < 2; h++)
            {
                __syncthreads(); // the previous half's epilogue has read buf
                // work items u = thread + 512 i (0 <= u <= 4096): the eight spectrum loads of an
                // item first, then its products
                for (int i0 = 0; i0 < 9; i0 += 1)
                {
                    double2 v[1][8];
#pragma unroll
                    for (int j = 0; j < 1; j++)
                    {
                        const int u = (int)threadIdx.x + kF2T * (i0 + j), u2 = u + kFPts;
                        if (u <= kFPts / 2)
                        {
                            v[j][0] = X[u];
                            v[j][1] = Y[u];
                            v[j][2] = X[N - u];
                            v[j][3] = Y[N - u];
                            v[j][4] = X[u2];
                            v[j][5] = Y[u2];
                            v[j][6] = X[N - u2];
                            v[j][7] = Y[N - u2];
                        }
                    }
#pragma unroll
                    for (int j = 0; j < 1; j++)
                    {
                        const int u = (int)threadIdx.x + kF2T * (i0 + j), u2 = u + kFPts;
                        if (u > kFPts / 2)
                            continue;
                        // C[u], C[N - u] from V[u], V[N - u]; C[u + 8192], C[8192 - u] from V[u + 8192], V[8192 - u]
                        const double2 V1 = cmul(v[j][0], v[j][1]), V1n = cmul(v[j][2], v[j][3]);
                        const double2 E1 = cadd(V1, conj2(V1n)), O1 = cmul(csub(V1, conj2(V1n)), root<1>(R, u));
                        const double2 Cu = cadd(E1, mul_si<1>(O1)), CNu = cadd(conj2(E1), mul_si<1>(conj2(O1)));
                        const double2 V2 = cmul(v[j][4], v[j][5]), V2n = cmul(v[j][6], v[j][7]);
                        const double2 E2 = cadd(V2, conj2(V2n)), O2 = cmul(csub(V2, conj2(V2n)), root<1>(R, u2));
                        const double2 Cv = cadd(E2, mul_si<1>(O2)), C8u = cadd(conj2(E2), mul_si<1>(conj2(O2)));
                        if (h == 0)
                        {
                            buf[pidx(u)] = cadd(Cu, Cv);
                            if (u > 0 && u < kFPts / 2)
                                buf[pidx(kFPts - u)] = cadd(C8u, CNu);
                        }
                        else
                        {
                            buf[pidx(u)] = cmul(csub(Cu, Cv), root<1>(R, 2 * u));
                            if (u > 0 && u < kFPts / 2)
                                buf[pidx(kFPts - u)] = cmul(csub(C8u, CNu), root<1>(R, 2 * (kFPts - u)));
                        }
                    }
                }
                __syncthreads();
                fft8192_r16<1>(buf, R);
                // work item u = it * 512 + thread of this half takes output k = (base >> 2) + u of
                // its transform, c[2 k + h] of the whole one, whose real and imaginary parts are
                // the dot products of windows o = 4 u - (base & 3) + 2 h and o + 1 (those in
                // [o_lo, o_hi)); u <= 4096 covers the piece's windows (o_hi <= 16384 keeps u, and
                // so k <= 8191, in bounds wherever a window is in range).
                for (int it = 0; it < 9; it++)
                {
                    if (it * kF2T + (int)(threadIdx.x & ~31u) >= kF3Items)
                        continue; // no item of this warp (uniform across the warp)
                    const int u = it * kF2T + (int)threadIdx.x;
                    const int o0 = 4 * u - (base & 3) + 2 * h;
                    float4 st[2];
                    bool inr[2], hit[2];
                    uint32_t jr[2];
                    float up[2], lo[2];
#pragma unroll
                    for (int j = 0; j < 2; j++)
                    {
                        inr[j] = u < kF3Items && o0 + j >= o_lo && o0 + j < o_hi;
                        jr[j] = (uint32_t)rel + (uint32_t)(o0 + j);
                    }
                    float4 *slot = cache + h * 2 * kF3Items + 2 * u;
                    if (cached)
                    {
#pragma unroll
                        for (int j = 0; j < 2; j++)
                            st[j] = inr[j] ? slot[j] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    }
                    else
                    {
                        WinIn w[2];
#pragma unroll
                        for (int j = 0; j < 2; j++)
                            w[j] = load_window(a, P.m, inr[j], (uint64_t)((int64_t)a.w0 + (int64_t)jr[j]));
#pragma unroll
                        for (int j = 0; j < 2; j++)
                        {
                            st[j] = fold_window(window_stats4(a, P.m, P.inv_m, inr[j],
                                                              (uint64_t)((int64_t)a.w0 + (int64_t)jr[j]), w[j]),
                                                c0, c1, P.m, shift, e_dot);
                            if (inr[j])
                                slot[j] = st[j];
                        }
                    }
                    double2 c = make_double2(0.0, 0.0);
                    if (inr[0] || inr[1])
                        c = final_out<1>(buf, R, (base >> 2) + u);
                    corr_eval(a, P, t, jr[0], st[0], c.x * inv_l, up[0], lo[0], hit[0]);
                    corr_eval(a, P, t, jr[1], st[1], c.y * inv_l, up[1], lo[1], hit[1]);
                    if (P.mode == TM_MODE_KNN)
                        bucket_minima<2>(a, t, lane, inr, jr, up, lo); // the warp spans 4 x 32 windows
                    else
#pragma unroll
                        for (int j = 0; j < 2; j++)
                            emit_hits(a, t, lane, hit[j], jr[j]);
                }
            }
            cached_m = P.m;
        }
    }
}

void fft_roots(double2 *host384)
{
    // R1[a] = e^{2 pi i a / 32768} (a < 128), R2[b] = e^{2 pi i 128 b / 32768} (b < 256), in
    // extended precision
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int a = 0; a < 128; a++)
    {
        const long double t = two_pi * (long double)a / 32768.0L;
        host384[a] = make_double2((double)cosl(t), (double)sinl(t));
    }
    for (int b = 0; b < 256; b++)
    {
        const long double t = two_pi * (long double)(128 * b) / 32768.0L;
        host384[128 + b] = make_double2((double)cosl(t), (double)sinl(t));
    }
}

uint32_t fft2_pieces(uint64_t n) { return (uint32_t)((n + kF2S - 1) / kF2S); }
uint32_t fft3_pieces(uint64_t n) { return (uint32_t)((n + kF3S - 1) / kF3S); }

cudaError_t launch_fft2_pieces(const float *clean, uint64_t n, const double *centres, uint32_t p0, uint32_t count,
                               const double2 *roots, double2 *X, double *shifts, double *norms, cudaStream_t s)
{
    cudaFuncSetAttribute(k_fft2_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kF2Smem);
    if (count > 0)
        k_fft2_forward<<<count, kF2T, kF2Smem, s>>>(clean, n, centres, p0, nullptr, nullptr, nullptr, roots,
                                                     X + (size_t)p0 * kF2H, shifts, norms);
    return cudaGetLastError();
}

cudaError_t launch_fft2_templates(const float *q, const TemplParam *tp, const int *rows, int nrows,
                                  const double2 *roots, double2 *Y, cudaStream_t s)
{
    cudaFuncSetAttribute(k_fft2_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kF2Smem);
    if (nrows > 0)
        k_fft2_forward<<<nrows, kF2T, kF2Smem, s>>>(nullptr, 0, nullptr, 0, q, tp, rows, roots, Y, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_fft2_corr(const Fft2Args &a, int sms, cudaStream_t s)
{
    cudaFuncSetAttribute(k_fft2_corr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kF2Smem);
    if (a.p_count > 0 && a.nrows > 0)
        k_fft2_corr<<<(unsigned)std::min<uint32_t>(a.p_count, (uint32_t)sms), kF2T, kF2Smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_fft3_pieces(const float *clean, uint64_t n, const double *centres, uint32_t p0, uint32_t count,
                               const double2 *roots, double2 *X, double *shifts, double *norms, double2 *scratch,
                               int blocks, cudaStream_t s)
{
    cudaFuncSetAttribute(k_fft3_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kF2Smem);
    if (count > 0)
        k_fft3_forward<<<(unsigned)std::min<uint32_t>(count, (uint32_t)blocks), kF2T, kF2Smem, s>>>(
            clean, n, centres, p0, count, nullptr, nullptr, nullptr, roots, X + (size_t)p0 * kF3H, shifts, norms,
            scratch);
    return cudaGetLastError();
}

cudaError_t launch_fft3_templates(const float *q, const TemplParam *tp, const int *rows, int nrows,
                                  const double2 *roots, double2 *Y, double2 *scratch, int blocks, cudaStream_t s)
{
    cudaFuncSetAttribute(k_fft3_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kF2Smem);
    if (nrows > 0)
        k_fft3_forward<<<(unsigned)std::min<int>(nrows, blocks), kF2T, kF2Smem, s>>>(
            nullptr, 0, nullptr, 0, (uint32_t)nrows, q, tp, rows, roots, Y, nullptr, nullptr, scratch);
    return cudaGetLastError();
}

cudaError_t launch_fft3_corr(const Fft2Args &a, int sms, cudaStream_t s)
{
    cudaFuncSetAttribute(k_fft3_corr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kF2Smem);
    if (a.p_count > 0 && a.nrows > 0)
        k_fft3_corr<<<(unsigned)std::min<uint32_t>(a.p_count, (uint32_t)sms), kF2T, kF2Smem, s>>>(a);
    return cudaGetLastError();
}

} // namespace tmb
