// FP32 FMA rate of the device: the denominator of the FP32 contraction kernel's roofline
// (the measured-peaks file carries a BF16 tensor figure and an HBM copy figure only).
// Every thread runs 8 independent FMA chains in registers (scalar FMAs, or 4 chains of
// packed pairs); 16 blocks of 256 threads per SM run as two waves of 64 resident warps (16
// per scheduler); the faster of the two forms is the rate.
#include "../../include/tremor_b200.h"

#include <cstdint>
#include <cuda_runtime.h>

namespace tmb {

constexpr int kProbeIters = 4096;

__global__ void __launch_bounds__(256) k_fma_probe(float seed, float *out)
{
    float a[8];
#pragma unroll
    for (int c = 0; c < 8; c++)
        a[c] = seed + 0.001f * (float)(threadIdx.x + c);
    const float b = 0.999999f, d = 1e-7f;
    for (int i = 0; i < kProbeIters; i++)
    {
#pragma unroll
        for (int c = 0; c < 8; c++)
            a[c] = fmaf(a[c], b, d);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < 8; c++)
        s += a[c];
    if (s == 12345.678f) // never true; keeps the chains live
        out[blockIdx.x] = s;
}

// The same with the packed FMA of sm_100 (fma.rn.f32x2: two FMAs per instruction), which
// the FP32 contraction uses: it needs half the issue slots for the same pipe work.
__global__ void __launch_bounds__(256) k_fma2_probe(float seed, float *out)
{
    uint64_t a[4];
#pragma unroll
    for (int c = 0; c < 4; c++)
    {
        const float lo = seed + 0.001f * (float)(threadIdx.x + 2 * c), hi = seed + 0.001f * (float)(threadIdx.x + 2 * c + 1);
        asm("mov.b64 %0, {%1, %2};" : "=l"(a[c]) : "f"(lo), "f"(hi));
    }
    uint64_t b, d;
    asm("mov.b64 %0, {%1, %1};" : "=l"(b) : "f"(0.999999f));
    asm("mov.b64 %0, {%1, %1};" : "=l"(d) : "f"(1e-7f));
    for (int i = 0; i < kProbeIters; i++)
    {
#pragma unroll
        for (int c = 0; c < 4; c++)
            asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(a[c]) : "l"(b), "l"(d));
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < 4; c++)
    {
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a[c]));
        s += lo + hi;
    }
    if (s == 12345.678f) // never true; keeps the chains live
        out[blockIdx.x] = s;
}

} // namespace tmb

extern "C" int tm_fp32_peak(int device, double *tflops)
{
    if (tflops == nullptr)
        return TM_ERR_ARGUMENT;
    int n = 0, sms = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
        return TM_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return TM_ERR_CUDA;
    float *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = TM_OK;
    if (cudaMalloc(&out, sizeof(float) * 4096) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess)
        rc = TM_ERR_CUDA;
    const int blocks = sms * 16;
    float best = 1e30f; // both probes do the same 8 FMA chains' work per thread: the faster counts
    for (int r = 0; rc == TM_OK && r < 10; r++)
    {
        cudaEventRecord(e0);
        if (r < 5)
            tmb::k_fma_probe<<<blocks, 256>>>(1.0f, out);
        else
            tmb::k_fma2_probe<<<blocks, 256>>>(1.0f, out);
        cudaEventRecord(e1);
        float ms = 0.0f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            rc = TM_ERR_CUDA;
        else if (r != 0 && r != 5 && ms < best) // the first launch of each warms up
            best = ms;
    }
    if (rc == TM_OK)
        *tflops = 2.0 * 8.0 * tmb::kProbeIters * static_cast<double>(blocks) * 256.0 / (best * 1e-3) / 1e12;
    if (out)
        cudaFree(out);
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    return rc;
}
