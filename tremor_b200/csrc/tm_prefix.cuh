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
    float mu;    // window mean (float)
    float iv;    // 1 / std (float)
    float estat; // bound on the distance error these statistics can cause (added to e)
};

// Statistics of window j (global start index) of length m. Returns 0 when the statistics
// are trustworthy, 2 when cancellation may have destroyed them (the window must then be
// re-scored exactly, whatever its distance). Pa = P[j], Pb = P[j + m].
//   var relative error  <= e_var / var   (prefix errors: gamma * sum of |terms| up to each end,
//                                          |sum (x - c)| <= sqrt(i * sum (x - c)^2))
//   std relative error  <= 0.5 e_var / var + rsqrtf's 2^-22 + float rounding
//   d error from stats  <= (4m + 2 |q| sqrt(m)) * (std rel. error) + 2 |sum q| * |mean error| / std
__device__ __forceinline__ int prefix_stats(double2 Pa, double2 Pb, uint64_t j, int m, double inv_m, double center,
                                            float qs, float s1q, WindowStats &w)
{
    const double s1 = Pb.x - Pa.x, s2 = Pb.y - Pa.y;
    const double mu_c = s1 * inv_m;
    const double var = s2 * inv_m - mu_c * mu_c;
    // var < 1e-22 (std < 1e-11): near the reference's 1e-12 cut, decided by the exact path
    if (!(var > 1e-22) || !(var < 1e36))
        return 2;
    // error terms in float with a 1.01 margin for their own rounding (they are bounds,
    // not values: a few ulps do not matter)
    const float fg = (float)kPrefixGamma * 1.01f, fe = (float)kEps64 * 1.01f, fm = (float)inv_m;
    const float a2 = (float)Pa.y, b2 = (float)Pb.y, fs2 = (float)s2, fmu = (float)mu_c;
    const float e_s2 = fg * (a2 + b2) + 4.0f * fe * fs2;
    const float e_s1 = fg * (sqrtf((float)j * a2) + sqrtf((float)(j + m) * b2)) * 1.001f + 4.0f * fe * fabsf((float)s1);
    const float e_var = (e_s2 + 2.0f * fabsf(fmu) * e_s1) * fm + 8.0f * fe * fs2 * fm;
    const float fvar = (float)var;
    if (e_var > 1e-4f * fvar)
        return 2;
    const double mu = mu_c + center;
    w.mu = (float)mu;
    w.iv = rsqrtf(fvar);
    const float rel_sd = 0.5f * e_var / fvar + 6.0e-7f;
    const float e_mu = e_s1 * fm + 6.0e-8f * fabsf(w.mu) + 4.0f * fe * fabsf(w.mu);
    w.estat = 1.25f * ((4.0f * (float)m + 2.0f * qs) * rel_sd + 2.0f * fabsf(s1q) * e_mu * w.iv);
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
