// tm_result_fp64: the error of every returned answer against FP64.
//
// The searches return the reference's FP32 distances bit for bit (ZnormSearch.hpp:103-165
// on float statistics and a float z-normalised template), so their error against an exact
// computation is the reference's own. This entry point states it per answer: the squared
// z-normalised distance of the same (template, window) recomputed entirely in FP64 from the
// raw samples, which the caller compares with the returned FP32 distance. The reference's
// own validation compares correlations with an FP64 implementation within 2e-4
// (experiments/validate_search.py:80-86, :127).
//
// FP64 distance of window p for template q (m samples):
//   template: mean and population std by two FP64 passes over the raw template, z-normalised
//             in FP64 (all zeros when std <= 1e-12, as znormalize_inplace);
//   window:   mean and population std by two FP64 passes over raw[p, p + m) with missing
//             samples (-100000) counted as 0 (SkipSequential.cpp:157-190, kept in FP64);
//   distance: sum over i of (qhat_i - (x_i - mean) / std)^2 in FP64 (+inf when the window's
//             std <= 1e-12, where the reference returns FLT_MAX).
// One warp per answer; FP64 sums over lanes, then a shuffle reduction.
#include <math_constants.h>

#include "tm_core.h"

namespace tmb {

__device__ __forceinline__ double warp_sum64(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void k_fp64_distance(const float *__restrict__ raw, uint64_t n, const double *__restrict__ qhat, int m,
                                const uint64_t *__restrict__ pos, const uint8_t *__restrict__ skip, uint64_t count,
                                double *__restrict__ out)
{
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= count)
        return;
    const uint64_t p = pos[warp];
    if (skip[warp] || p + static_cast<uint64_t>(m) > n)
    {
        if (lane == 0)
            out[warp] = skip[warp] ? CUDART_INF : CUDART_NAN;
        return;
    }
    const float *w = raw + p;
    auto clean = [](float v) { return v == kMissing ? 0.0 : static_cast<double>(v); };
    double s = 0.0;
    for (int i = lane; i < m; i += 32)
        s += clean(w[i]);
    const double mean = warp_sum64(s) / m;
    double s2 = 0.0;
    for (int i = lane; i < m; i += 32)
    {
        const double v = clean(w[i]) - mean;
        s2 = fma(v, v, s2);
    }
    const double sd = sqrt(warp_sum64(s2) / m);
    if (sd <= 1e-12)
    {
        if (lane == 0)
            out[warp] = CUDART_INF;
        return;
    }
    const double inv = 1.0 / sd;
    double d = 0.0;
    for (int i = lane; i < m; i += 32)
    {
        const double diff = qhat[i] - (clean(w[i]) - mean) * inv;
        d = fma(diff, diff, d);
    }
    d = warp_sum64(d);
    if (lane == 0)
        out[warp] = d;
}

} // namespace tmb

using namespace tmh;

extern "C" int tm_result_fp64(tm_ctx *ctx, const tm_result *res, int request, const float *templ, int m,
                              double *d64, uint64_t capacity)
{
    if (ctx == nullptr || res == nullptr || templ == nullptr || m < 1 || request < 0 ||
        request >= static_cast<int>(res->answers.size()) || (capacity > 0 && d64 == nullptr))
        return TM_ERR_ARGUMENT;
    if (static_cast<uint64_t>(m) > ctx->n)
        return TM_ERR_ARGUMENT;
    return guarded(ctx, [&] {
        TM_CUDA(cudaSetDevice(ctx->device));
        const Answer &a = res->answers[request];
        const uint64_t count = std::min<uint64_t>(a.size(), capacity);
        if (count == 0)
            return;
        // the template, z-normalised in FP64 (two passes)
        std::vector<double> q(static_cast<size_t>(m));
        double sum = 0.0;
        for (int i = 0; i < m; i++)
            sum += static_cast<double>(templ[i]);
        const double mean = sum / m;
        double sq = 0.0;
        for (int i = 0; i < m; i++)
        {
            const double v = static_cast<double>(templ[i]) - mean;
            sq += v * v;
        }
        const double sd = std::sqrt(sq / m);
        for (int i = 0; i < m; i++)
            q[i] = sd <= 1e-12 ? 0.0 : (static_cast<double>(templ[i]) - mean) / sd;
        std::vector<uint64_t> pos(count);
        std::vector<uint8_t> skip(count);
        for (uint64_t i = 0; i < count; i++)
        {
            const Hit h = a.at(i);
            pos[i] = h.pos;
            skip[i] = h.dist >= FLT_MAX ? 1 : 0; // padding and constant windows: +inf
        }
        Lane &L = ctx->main;
        cudaStream_t s = L.stream;
        DevBuf dq, dp, ds, dout;
        dq.reserve_on(sizeof(double) * m, s, ctx->pool);
        dp.reserve_on(sizeof(uint64_t) * count, s, ctx->pool);
        ds.reserve_on(count, s, ctx->pool);
        dout.reserve_on(sizeof(double) * count, s, ctx->pool);
        TM_CUDA(cudaMemcpyAsync(dq.p, q.data(), sizeof(double) * m, cudaMemcpyHostToDevice, s));
        TM_CUDA(cudaMemcpyAsync(dp.p, pos.data(), sizeof(uint64_t) * count, cudaMemcpyHostToDevice, s));
        TM_CUDA(cudaMemcpyAsync(ds.p, skip.data(), count, cudaMemcpyHostToDevice, s));
        const uint64_t threads = count * 32;
        const unsigned blocks = static_cast<unsigned>((threads + 255) / 256);
        tmb::k_fp64_distance<<<blocks, 256, 0, s>>>(ctx->raw.as<float>(), ctx->n, dq.as<double>(), m,
                                                    dp.as<uint64_t>(), ds.as<uint8_t>(), count, dout.as<double>());
        TM_CUDA(cudaGetLastError());
        count_launch(L);
        TM_CUDA(cudaMemcpyAsync(d64, dout.p, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
        // stream-ordered frees after the copy back
        for (DevBuf *b : {&dq, &dp, &ds, &dout})
            b->release_on(s);
        TM_CUDA(cudaStreamSynchronize(s));
    });
}
