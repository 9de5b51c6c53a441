// Window statistics of any length from the resident block-local FP64 prefix sums
// (tm_prefix.cu), with a bound on their error, for contraction tiles that mix template
// lengths.
#pragma once

#include "tm_internal.cuh"

namespace tmb {

constexpr int kPrefixBlockLog = 16;
constexpr uint64_t kPrefixBlock = 1ull << kPrefixBlockLog; // samples per prefix block (>= any mixed length)

// Bound on the accumulated error of one prefix sum, relative to the sum of magnitudes
// it covers: a sample passes through at most ~25 additions (8 per thread, 5 + 5 shuffle
// levels, the 8 chunk totals of its block) plus its own centring and squaring; 80 units
// leave a wide margin.
constexpr double kPrefixGamma = 80.0 * 1.1102230246251565e-16;
constexpr double kEps64 = 1.1102230246251565e-16;

// The resident prefix sums: Q[i] (block-local, n + 1 entries), T[b] and C[b] (block
// totals and centres, one more entry than there are blocks).
struct PrefixView
{
    const double2 *Q;
    const double2 *T;
    const double *C;
};

struct WindowStats
{
    float mu;     // window mean (float)
    float iv;     // 1 / std (float)
    float rel_sd; // bound on the relative error of the std
    float e_mu;   // bound on the absolute error of the mean
};

// An upper bound on sqrt(x) for x >= 0 (0 for x = 0) from the fast reciprocal square root:
// its relative error is below 2^-21, so the factor 1 + 2^-19 keeps the result above sqrt(x).
// For the error-bound terms only (never for a value).
__device__ __forceinline__ float sqrt_up(float x)
{
    return x > 0.0f ? x * rsqrtf(x) * (1.0f + 1.9073486e-06f) : 0.0f;
}

// Bound on the distance error that statistics with these error bounds can cause, for a
// template of length m with |q| sqrt(m) = qs and sum q = s1q (added to e).
__device__ __forceinline__ float stats_error(const WindowStats &w, int m, float qs, float s1q)
{
    return 1.25f * ((4.0f * (float)m + 2.0f * qs) * w.rel_sd + 2.0f * fabsf(s1q) * w.e_mu * w.iv);
}

// A window's first and second sums relative to its start block's centre, with bounds on
// their errors (the two cases of window_prefix_stats).
struct PrefixSums
{
    double s1, s2;
    float e_s1, e_s2;
};

// The window lies in one prefix block: na and nb are the block offsets of its start and
// end, qa = (float) Qa.y.
__device__ __forceinline__ PrefixSums prefix_sums_one_block(double2 Qa, double2 Qb, float na, float nb, float qa)
{
    const float fg = (float)kPrefixGamma * 1.01f;
    const float qb = (float)Qb.y;
    PrefixSums r;
    r.s1 = Qb.x - Qa.x;
    r.s2 = Qb.y - Qa.y;
    r.e_s2 = fg * (qa + qb);
    // sqrt(na qa) + sqrt(nb qb) <= sqrt(2 (na qa + nb qb)) (Cauchy-Schwarz)
    r.e_s1 = 1.001f * fg * sqrt_up(2.0f * (na * qa + nb * qb));
    return r;
}

// The window starts in block b1 and ends in block be = b1 + 1 (m <= kPrefixBlock).
__device__ __forceinline__ PrefixSums prefix_sums_two_blocks(const PrefixView &pv, double2 Qa, double2 Qb, uint64_t j,
                                                             int m)
{
    const uint64_t e = j + (uint64_t)m;
    const uint64_t b1 = j >> kPrefixBlockLog, be = e >> kPrefixBlockLog;
    const float fg = (float)kPrefixGamma * 1.01f, fe = (float)kEps64 * 1.01f;
    const float na = (float)(j - (b1 << kPrefixBlockLog)), qa = (float)Qa.y, qb = (float)Qb.y;
    const double2 t = pv.T[b1];
    const double d = pv.C[be] - pv.C[b1];
    const double n2 = (double)(e - (be << kPrefixBlockLog));
    PrefixSums r;
    r.s1 = (t.x - Qa.x) + (Qb.x + n2 * d);
    r.s2 = (t.y - Qa.y) + (Qb.y + (2.0 * d * Qb.x + n2 * d * d));
    const float tq = (float)t.y, fd = fabsf((float)d), fn2 = (float)n2, q1b = fabsf((float)Qb.x);
    const float nt = (float)kPrefixBlock;
    const float eq1b = 1.001f * fg * sqrt_up(fn2 * qb);
    r.e_s2 = fg * (tq + qa + qb) + 2.0f * fd * eq1b + 8.0f * fe * (2.0f * fd * q1b + fn2 * fd * fd) +
             4.0f * fe * fd * (q1b + fn2 * fd);
    r.e_s1 = 1.001f * fg * sqrt_up(2.0f * (nt * tq + na * qa)) + eq1b + 4.0f * fe * fn2 * fd +
             4.0f * fe * (fabsf((float)t.x) + fabsf((float)Qa.x) + q1b + fn2 * fd);
    return r;
}

// The statistics from a window's sums (centre c of its start block): 0 when trustworthy,
// 2 when cancellation may have destroyed them (w is then meaningless). Branch-free apart
// from its result, so that callers can evaluate several windows side by side.
__device__ __forceinline__ int prefix_stats_tail(PrefixSums ps, int m, double inv_m, double c, WindowStats &w)
{
    const float fe = (float)kEps64 * 1.01f;
    const double mu_c = ps.s1 * inv_m;
    const double var = fma(-mu_c, mu_c, ps.s2 * inv_m);
    const float fvar = (float)var, fmu = (float)mu_c;
    // 1 / m from the caller's FP64 inverse, rounded up (a factor for the bounds only)
    const float fm = (float)m, fim = (float)inv_m * (1.0f + 1.1920929e-07f);
    const float fs2 = fm * (fvar + fmu * fmu) * 1.0001f;
    const float e_s2 = ps.e_s2 + 4.0f * fe * fs2;
    const float e_s1 = ps.e_s1 + 4.0f * fe * fm * fabsf(fmu);
    const float e_var = (e_s2 + 2.0f * fabsf(fmu) * e_s1 + 8.0f * fe * fs2) * fim * 1.0001f;
    const float center_f = (float)c;
    w.iv = rsqrtf(fvar);
    w.mu = fmu + center_f;
    w.rel_sd = 0.5f * e_var * w.iv * w.iv * 1.001f + 6.0e-7f;
    w.e_mu = e_s1 * fim + 1.2e-7f * (fabsf(w.mu) + fabsf(center_f)) + 4.0f * fe * fabsf(w.mu) +
             6.0e-8f * fabsf(center_f);
    // var < 1e-22 (std < 1e-11): near the reference's 1e-12 cut, decided by the exact path
    return (var > 1e-22 && var < 1e36 && e_var <= 1e-4f * fvar) ? 0 : 2;
}

// Fast path for windows that lie in one prefix block and are well conditioned (most of
// them): bounds that hold for every single-block window of block b, from its block total of
// squares T2 (the block-local prefix of squares only grows, so qa, qb <= T2 up to rounding,
// and na, nb <= 2^16):
//   e_s2 = fg (qa + qb)                        <= a = 2 fg T2
//   e_s1 = 1.001 fg sqrt(2 (na qa + nb qb))    <= b = 1.001 fg 512 sqrt(T2)
// (each with a 1e-5 margin). When, in addition, (a + 2 |mu_c| b) / m <= 0.9e-7 var and
// mu_c^2 <= 1e6 var, prefix_stats_tail's e_var is at most 1.0004e-7 var, so the statistics
// are trusted and its rel_sd is at most 0.5 x 1.0004e-7 (1 + 2^-21) 1.001 + 6e-7 < 6.6e-7
// (kFastRelSd), and its e_mu is at most b / m + 1.3e-7 |mu| + 1.9e-7 |c|. mu and 1 / std are
// computed exactly as there.
struct BlockBounds
{
    float a, b;
};

constexpr float kFastRelSd = 6.6e-7f;

__device__ __forceinline__ BlockBounds block_bounds(double t2)
{
    const float fg = (float)kPrefixGamma * 1.01f;
    const float T = (float)t2 * 1.00001f;
    return BlockBounds{2.0f * fg * T * 1.00001f, 1.001f * fg * 512.0f * sqrt_up(T) * 1.00001f};
}

// Returns true when the fast path applies (the window must lie in one block); then mu, iv
// are the window's mean and 1 / std, e_mu a bound on the error of mu, and kFastRelSd one on
// the relative error of the std. fim: (float) inv_m rounded up, cf: (float) c.
__device__ __forceinline__ bool prefix_stats_fast(double2 Qa, double2 Qb, double inv_m, float fim, float cf,
                                                  BlockBounds bb, float &mu, float &iv, float &e_mu)
{
    const double s1 = Qb.x - Qa.x, s2 = Qb.y - Qa.y;
    const double mu_c = s1 * inv_m;
    const double var = fma(-mu_c, mu_c, s2 * inv_m);
    const float fvar = (float)var, fmu = (float)mu_c;
    iv = rsqrtf(fvar);
    mu = fmu + cf;
    e_mu = bb.b * fim + 1.3e-7f * fabsf(mu) + 1.9e-7f * fabsf(cf);
    return fvar > 2e-22f && fvar < 1e36f && fmu * fmu <= 1e6f * fvar &&
           (bb.a + 2.0f * fabsf(fmu) * bb.b) * fim <= 0.9e-7f * fvar;
}

// Statistics of window [j, j + m) (global sample index, m <= kPrefixBlock) from its
// block-local prefix sums Qa = Q[j], Qb = Q[j + m]. Returns 0 when they are trustworthy, 2
// when cancellation may have destroyed them (the window must then be re-scored exactly,
// whatever its distance).
//   One block b:  s = Qb - Qa, centre c_b.
//   Two blocks b, b + 1 (the window ends in b + 1 after n2 samples):
//     s1 = (T1[b] - Qa1) + (Qb1 + n2 d),  s2 = (T2[b] - Qa2) + (Qb2 + 2 d Qb1 + n2 d^2),
//     d = c_{b+1} - c_b: the second block's part re-centred on c_b.
// Error bounds: a prefix value's error is at most gamma x the sum of |terms| it covers;
// for the squares that is the value itself, for the first sums at most sqrt(count x the
// squares); the re-centring adds the error of Qb1 times 2|d| and the roundings of its
// products. The bounds are evaluated in float with margins (bounds, not values).
//   var relative error  <= e_var / var
//   std relative error  <= 0.5 e_var / var + rsqrtf's 2^-22 + float rounding
__device__ __forceinline__ int window_prefix_stats(const PrefixView &pv, double2 Qa, double2 Qb, uint64_t j, int m,
                                                   double inv_m, WindowStats &w)
{
    const uint64_t e = j + (uint64_t)m;
    const uint64_t b1 = j >> kPrefixBlockLog, be = e >> kPrefixBlockLog;
    PrefixSums ps;
    if (be == b1)
        ps = prefix_sums_one_block(Qa, Qb, (float)(j - (b1 << kPrefixBlockLog)),
                                   (float)(e - (b1 << kPrefixBlockLog)), (float)Qa.y);
    else
        ps = prefix_sums_two_blocks(pv, Qa, Qb, j, m);
    return prefix_stats_tail(ps, m, inv_m, pv.C[b1], w);
}

// fast_distance (tm_epilogue.cuh) for statistics from prefix sums: the a4 term of the
// per-length statistics is replaced by the window's own estat.
__device__ __forceinline__ void fast_distance_mixed(const TemplParam &p, float a1, float dot, float mu, float iv,
                                                    float shift, float estat, float &d, float &e)
{
    const float ms = mu - shift;
    const float cross = (dot - ms * p.s1) * iv;
    d = p.c_lin - 2.0f * cross;
    const float r = ms * iv, r0 = mu * iv;
    e = a1 * sqrtf(1.0f + r * r) + p.a2 + p.a3 * fmaxf(d, 0.0f) + p.a5 * r0 * r0 +
        p.a6 * (fabsf(mu) + fabsf(shift)) * iv + estat;
}

} // namespace tmb
