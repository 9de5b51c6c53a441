// Internal declarations shared by the tremor_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace tmb {

constexpr float kMissing = -100000.0f; // ZnormSearch.hpp:21
constexpr float kFltMax = 3.402823466e+38f;
constexpr int kZnormBlock = 32;      // ZnormSearch.hpp:65
constexpr int kBucket = 2048;        // windows per kNN bound bucket
constexpr int kStagePad = 16384 + 512; // zero samples after the waveform (template padding)

// per-window flags (one byte per window and length)
constexpr uint8_t kFlagMissingStart = 1; // first sample missing: not searched
constexpr uint8_t kFlagDegenerate = 2;   // reference std <= 1e-12: distance FLT_MAX
constexpr uint8_t kFlagNeedsExact = 4;   // prefix-sum statistics not trusted: two-pass fix-up
constexpr uint8_t kFlagExact = 8;        // statistics are the reference's two-pass values

// Per-template constants of the fused epilogue (one per template in a batch).
struct TemplParam
{
    double inv_m;  // 1 / m (statistics from prefix sums)
    float s1;      // sum of z-normalised template samples
    float c_lin;   // sum q^2 + m
    float thr_ed;  // threshold mode: cc_to_ed(correlation, m); kNN: unused
    float a1_main; // error-bound coefficients, see fast_distance (tm_epilogue.cuh);
    float a1_fp32; //   a1 for the main contraction kernel and for the FP32 re-pass
    float a2, a3, a4, a5, a6;
    int mode;         // TM_MODE_KNN (1) / TM_MODE_THRESHOLD (0)
    int m;            // template length
    int k;            // kNN answers
    int merge;        // merge offset
    int64_t q_offset; // float offset of the template in the packed template array
    int64_t order_offset; // int offset of its block order
    uint32_t wcount;  // windows of this template in the searched range (mixed-length tiles)
    float qs;         // |q| sqrt(m)
};

// A tile of a mixed-length group (128 template rows, or a column tile): its K extent.
struct TileInfo
{
    int kb; // K blocks of 64 samples (the longest template of the tile)
};

// A candidate window for exact re-scoring: template slot and window index relative
// to the window range start, plus (after re-scoring) the reference FP32 distance.
struct Candidate
{
    uint32_t templ;
    uint32_t window;
};

// Monotone map float -> uint32 so that unsigned min equals float min.
__host__ __device__ inline uint32_t float_key(float f)
{
    uint32_t b;
#ifdef __CUDA_ARCH__
    b = __float_as_uint(f);
#else
    __builtin_memcpy(&b, &f, 4);
#endif
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float key_float(uint32_t k)
{
    uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
#ifdef __CUDA_ARCH__
    f = __uint_as_float(b);
#else
    __builtin_memcpy(&f, &b, 4);
#endif
    return f;
}
constexpr uint32_t kEmptyKey = 0xffffffffu; // above every finite float's key
__host__ __device__ inline float inf_f()
{
#ifdef __CUDA_ARCH__
    return __int_as_float(0x7f800000);
#else
    return __builtin_huge_valf();
#endif
}

} // namespace tmb
