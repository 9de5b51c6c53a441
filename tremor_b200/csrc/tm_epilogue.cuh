// Fused distance epilogue shared by the contraction kernels.
#pragma once

#include "tm_internal.cuh"

namespace tmb {

// Arguments of a contraction launch over windows [w0, w0 + W) of one length m.
struct ScanArgs
{
    const float *x;        // clean waveform (missing -> 0), global sample index, zero padded
    const float *q;        // z-normalised templates, T_pad x m_pad, zero padded
    const TemplParam *tp;  // T_pad
    const float *mean;     // [W] window means
    const float *inv;      // [W] 1 / std; 0 for windows that are not searched
    uint64_t w0;
    uint32_t W;
    int m_pad;
    int T;
    uint32_t *bmin_u;      // [T][nb] bucket minima of d + E (float keys)
    uint32_t *bmin_l;      // [T][nb] bucket minima of d - E
    uint32_t nb;
    Candidate *cand;
    uint32_t *cand_count;
    uint32_t cand_cap;
    const void *q_hi;      // tensor-core kernel: BF16 high and low halves of q, t_rows x m_pad
    const void *q_lo;
    int t_rows;
    int *err;              // set (non-zero) by a kernel that gave up waiting
    float *dbg_d;          // diagnostics (tm_bound_diagnostics): every d and its bound e,
    float *dbg_e;          //   [T][W]; null in searches
    // templates of several lengths in one tile (statistics from prefix sums, tm_prefix.cu)
    const float *raw;      // raw waveform (missing first samples)
    const double2 *P;      // block-local FP64 prefix sums Q, n + 1 (tm_prefix.cu)
    const double2 *PT;     //   their block totals
    const double *PC;      //   and block centres
    const uint16_t *run;   // constant-run lengths
    const TileInfo *tiles; // mixed lengths: per tile, its K blocks
    int k_stride;          // row stride of the template arrays
    uint64_t n;            // samples of the waveform (P has n + 1 entries)
    int col_tile;          // window-major kernel: templates per column tile (32, 64, 128); 0: row tiles
    float *qt;             // FP32 kernel: scratch for the templates by 64-template tile, [tile][m_pad][64]
                           //   (T_pad x m_pad floats; filled by launch_scan_fp32 from q)
};

// Distance d of one (template, window) pair from its shifted dot product
// dot = sum_i q_i (x_{j+i} - shift), and the bound e >= |d - reference FP32 distance|.
//
// The terms of e (u = 2^-24, qs = |q| sqrt(m), r = (mu - shift) / sigma, r0 = mu / sigma):
//   a1 sqrt(1+r^2): error of dot (accumulation chain gamma, shift rounding) and of the
//                   final float evaluation, |sum |q||x - shift|| <= qs sigma sqrt(1+r^2);
//   a2:             1/sigma rounding on the cross term, the reference's own cross-term
//                   and sum-of-squares rounding, final rounding of q2 + m;
//   a3 max(d,0):    the reference's accumulation (m/16 + 4 roundings per term, then the
//                   tail), ZnormSearch.hpp:134-163;
//   a4 (1+2 r0^2):  error of the FP64 segmented-sum statistics;
//   a5 r0^2:        rounding of the mean to float inside sum (x - mu_f)^2 / sigma_f^2;
//   a6:             rounding of the mean times sum q.
// All coefficients carry a 1.25 safety factor (host side, tm_host.cpp).
__device__ __forceinline__ void fast_distance(const TemplParam &p, float a1, float dot, float mu, float iv,
                                              float shift, float &d, float &e)
{
    const float ms = mu - shift;
    const float cross = (dot - ms * p.s1) * iv;
    d = p.c_lin - 2.0f * cross;
    const float r = ms * iv, r0 = mu * iv;
    e = a1 * sqrtf(1.0f + r * r) + p.a2 + p.a3 * fmaxf(d, 0.0f) + p.a4 * (1.0f + 2.0f * r0 * r0) +
        p.a5 * r0 * r0 + p.a6 * (fabsf(mu) + fabsf(shift)) * iv;
}

// Warp-aggregated append of the windows j0 + w (bit w of mask) of template t.
// Every lane of the warp must call it. Entries past the capacity are counted, not written.
__device__ __forceinline__ void emit_candidates(uint32_t mask, int lane, uint32_t t, uint32_t j0, Candidate *cand,
                                                uint32_t *count, uint32_t cap)
{
    const int c = __popc(mask);
    int incl = c;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off)
            incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0)
        return;
    uint32_t base = 0;
    if (lane == 31)
        base = atomicAdd(count, (uint32_t)total);
    base = __shfl_sync(0xffffffffu, base, 31);
    uint32_t pos = base + (uint32_t)(incl - c);
    while (mask)
    {
        const int w = __ffs(mask) - 1;
        mask &= mask - 1;
        if (pos < cap)
            cand[pos] = Candidate{t, j0 + (uint32_t)w};
        pos++;
    }
}

// Per-warp staging of candidates in shared memory: a warp appends to its own buffer and
// reserves global slots with one atomicAdd per flush instead of one per emission, so many
// warps emitting at once do not serialise on the global counter. `n` is warp-uniform.

__device__ __forceinline__ void stage_flush(Candidate *sbuf, uint32_t &n, int lane, Candidate *cand, uint32_t *count,
                                            uint32_t cap)
{
    if (n == 0)
        return;
    uint32_t base = 0;
    if (lane == 0)
        base = atomicAdd(count, n);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (uint32_t i = lane; i < n; i += 32)
        if (base + i < cap)
            cand[base + i] = sbuf[i];
    __syncwarp();
    n = 0;
}

// One candidate per lane (template t, window j) where `hit`, through the warp's staging
// buffer (every lane must call it; kStageCap >= 32).
template <uint32_t kStageCap>
__device__ __forceinline__ void stage_emit_lane(bool hit, int lane, uint32_t t, uint32_t j, Candidate *sbuf,
                                                uint32_t &n, Candidate *cand, uint32_t *count, uint32_t cap)
{
    static_assert(kStageCap >= 32, "a warp's hits must fit the staging buffer");
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (b == 0u)
        return;
    const uint32_t total = (uint32_t)__popc(b);
    if (n + total > kStageCap)
        stage_flush(sbuf, n, lane, cand, count, cap);
    if (hit)
        sbuf[n + (uint32_t)__popc(b & ((1u << lane) - 1u))] = Candidate{t, j};
    __syncwarp();
    n += total;
}

// emit_candidates through the warp's staging buffer (every lane must call it).
template <uint32_t kStageCap>
__device__ __forceinline__ void stage_emit(uint32_t mask, int lane, uint32_t t, uint32_t j0, Candidate *sbuf,
                                           uint32_t &n, Candidate *cand, uint32_t *count, uint32_t cap)
{
    const int c = __popc(mask);
    int incl = c;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off)
            incl += v;
    }
    const uint32_t total = (uint32_t)__shfl_sync(0xffffffffu, incl, 31);
    if (total == 0)
        return;
    if (total > kStageCap)
    {
        emit_candidates(mask, lane, t, j0, cand, count, cap); // rare: more than a buffer at once
        return;
    }
    if (n + total > kStageCap)
        stage_flush(sbuf, n, lane, cand, count, cap);
    uint32_t pos = n + (uint32_t)(incl - c);
    while (mask)
    {
        const int w = __ffs(mask) - 1;
        mask &= mask - 1;
        sbuf[pos++] = Candidate{t, j0 + (uint32_t)w};
    }
    __syncwarp();
    n += total;
}

} // namespace tmb
