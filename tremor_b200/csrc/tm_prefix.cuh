// Window statistics of any length from the resident FP64 prefix sums (tm_prefix.cu),
// with a bound on their error, for contraction tiles that mix template lengths.
#pragma once

#include "tm_internal.cuh"

namespace tmb {

// Bound on the accumulated error of one prefix sum, relative to the sum of magnitudes
// it covers: a sample passes through at most ~40 additions (8 per thread, 5 + 5 shuffle
// levels, 5 + 5 + 5 levels for the chunk totals); doubled for margin.
constexpr double kPrefixGamma = 80.0 * 1.1102230246251565e-16;
constexpr double kEps64 = 1.1102230246251565e-16;

struct WindowStats
{
    float mu;     // window mean (float)
    float iv;     // 1 / std (float)
    float rel_sd; // bound on the relative error of the std
    float e_mu;   // bound on the absolute error of the mean
};

// Bound on the distance error that statistics with these error bounds can cause, for a
// template of length m with |q| sqrt(m) = qs and sum q = s1q (added to e).
__device__ __forceinline__ float stats_error(const WindowStats &w, int m, float qs, float s1q)
{
    return 1.25f * ((4.0f * (float)m + 2.0f * qs) * w.rel_sd + 2.0f * fabsf(s1q) * w.e_mu * w.iv);
}

// Statistics of window j (global start index) of length m (independent of the template).
// Returns 0 when the statistics are trustworthy, 2 when cancellation may have destroyed them (the window must then be
// re-scored exactly, whatever its distance). Pa = P[j] (a2 = (float)Pa.y), Pb = P[j + m].
//   prefix errors: gamma * (sum of |terms| up to each end); sum (x - c)^2 up to i is P2[i],
//   and sum |x - c| up to i <= sqrt(i * P2[i]) <= sqrt((j + m) * P2[j + m]) for i <= j + m
//   var relative error  <= e_var / var
//   std relative error  <= 0.5 e_var / var + rsqrtf's 2^-22 + float rounding
// The error terms are evaluated in float with margins (they are bounds, not values).
__device__ __forceinline__ int prefix_stats(double2 Pa, float a2, double2 Pb, uint64_t j, int m, double inv_m,
                                            float center_f, WindowStats &w)
{
    const double s1 = Pb.x - Pa.x, s2 = Pb.y - Pa.y;
    const double mu_c = s1 * inv_m;
    const double var = fma(-mu_c, mu_c, s2 * inv_m);
    // var < 1e-22 (std < 1e-11): near the reference's 1e-12 cut, decided by the exact path
    if (!(var > 1e-22) || !(var < 1e36))
        return 2;
    const float fvar = (float)var, fmu = (float)mu_c, fb2 = (float)Pb.y;
    const float fm = (float)m, fim = 1.0f / fm;
    const float fg = (float)kPrefixGamma * 1.01f, fe = (float)kEps64 * 1.01f;
    const float fs2 = fm * (fvar + fmu * fmu) * 1.0001f;
    const float e_s2 = fg * (a2 + fb2) + 4.0f * fe * fs2;
    const float e_s1 = 2.002f * fg * sqrtf((float)(j + (uint64_t)m) * fb2) + 4.0f * fe * fm * fabsf(fmu);
    const float e_var = (e_s2 + 2.0f * fabsf(fmu) * e_s1 + 8.0f * fe * fs2) * fim * 1.0001f;
    if (e_var > 1e-4f * fvar)
        return 2;
    w.iv = rsqrtf(fvar);
    w.mu = fmu + center_f;
    w.rel_sd = 0.5f * e_var * w.iv * w.iv * 1.001f + 6.0e-7f;
    w.e_mu = e_s1 * fim + 1.2e-7f * (fabsf(w.mu) + fabsf(center_f)) + 4.0f * fe * fabsf(w.mu);
    return 0;
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
