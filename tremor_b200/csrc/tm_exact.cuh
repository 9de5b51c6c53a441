// The reference's exact arithmetic, restated on the device operation by operation
// with round-to-nearest intrinsics (which the compiler neither contracts nor
// reorders), so the results are bit-identical to the reference built with
// g++ -O2 -mfma (GCC fuses a*b+c in C++ by default):
//   exact_stats       SkipSequential.cpp:243-259 (= indexing.cpp:128-152)
//   replica_distance  l2_dist_znorm_subsequence, ZnormSearch.hpp:103-165, without the
//                     early abandon (abandoning never changes the distance of a window
//                     that ends up in an answer set: partial sums only grow)
#pragma once

#include "tm_internal.cuh"

namespace tmb {

__device__ __forceinline__ float clean32(float v) { return v == kMissing ? 0.0f : v; }

// Two-pass FP64 mean and population std of window g, rounded to float; std <= 1e-12 -> 0.
__device__ __forceinline__ void exact_stats(const float *__restrict__ raw, uint64_t g, int m, float &mean_f,
                                            float &std_f)
{
    const float *w = raw + g;
    double sum = 0.0;
    for (int d = 0; d < m; d++)
        sum = __dadd_rn(sum, (double)clean32(w[d]));
    const double mean = __ddiv_rn(sum, (double)m);
    double squares = 0.0;
    for (int d = 0; d < m; d++)
    {
        const double c = __dsub_rn((double)clean32(w[d]), mean);
        squares = __fma_rn(c, c, squares);
    }
    const double sd = __dsqrt_rn(__ddiv_rn(squares, (double)m));
    mean_f = __double2float_rn(mean);
    std_f = sd <= 1e-12 ? 0.0f : __double2float_rn(sd);
}

// Squared z-normalised ED of the z-normalised template q against window g: 32-sample
// blocks in `order`, lanes l of two 8-wide accumulators (acc0 for samples i..i+7,
// acc1 for i+8..i+15 of each 16-sample step), horizontal sum in hsum256's order
// (ZnormSearch.hpp:92-97), then the m % 32 tail sequentially.
__device__ __forceinline__ float replica_distance(const float *__restrict__ q, const int *__restrict__ order,
                                                  const float *__restrict__ raw, uint64_t g, int m, float mean,
                                                  float stddev)
{
    if (stddev <= 1e-12f)
        return kFltMax;
    const float *x = raw + g;
    const float inv = __fdiv_rn(1.0f, stddev);
    float acc0[8], acc1[8];
#pragma unroll
    for (int l = 0; l < 8; l++)
        acc0[l] = acc1[l] = 0.0f;
    const int blocks = m / kZnormBlock;
    for (int b = 0; b < blocks; b++)
    {
        const int off = order[b];
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const int i = off + 16 * h;
#pragma unroll
            for (int l = 0; l < 8; l++)
            {
                const float r0 = clean32(x[i + l]), r1 = clean32(x[i + 8 + l]);
                const float d0 = __fmaf_rn(-__fsub_rn(r0, mean), inv, q[i + l]);
                const float d1 = __fmaf_rn(-__fsub_rn(r1, mean), inv, q[i + 8 + l]);
                acc0[l] = __fmaf_rn(d0, d0, acc0[l]);
                acc1[l] = __fmaf_rn(d1, d1, acc1[l]);
            }
        }
    }
    float v[8];
#pragma unroll
    for (int l = 0; l < 8; l++)
        v[l] = __fadd_rn(acc0[l], acc1[l]);
    const float s0 = __fadd_rn(v[0], v[4]), s1 = __fadd_rn(v[1], v[5]);
    const float s2 = __fadd_rn(v[2], v[6]), s3 = __fadd_rn(v[3], v[7]);
    float dist = __fadd_rn(__fadd_rn(s0, s2), __fadd_rn(s1, s3));
    for (int i = blocks * kZnormBlock; i < m; i++)
    {
        const float diff = __fmaf_rn(-__fsub_rn(clean32(x[i]), mean), inv, q[i]);
        dist = __fmaf_rn(diff, diff, dist);
    }
    return dist;
}

} // namespace tmb
