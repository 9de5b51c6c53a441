// tm_window_stats_noalloc: the window statistics of a device-resident waveform,
// computed without allocating any memory.
//
// Who needs it: callers that must not call cudaMalloc. A station-side detector that
// matches every new chunk of a live waveform within a fixed latency budget cannot
// afford cudaMalloc/cudaFree, which may synchronise the whole device and take
// unbounded time; a host runtime that hands all free device memory to its own pool
// allocator (PyTorch's caching allocator, for one) leaves nothing for an outside
// cudaMalloc. Such a caller owns its input and output buffers and passes them in.
//
// What it computes: for every window j of length m of raw[0..n), the statistics the
// reference keeps (SkipSequential.cpp:157-190): float mean and population std, (0, 0)
// when the window's first sample is missing (-100000), std 0 for constant windows
// (std <= 1e-12), and the flags byte of the searches (bit 0 missing first sample, bit 1
// constant, bit 3 two-pass statistics). The sums come from FP64 segmented suffix and
// prefix sums over segments of m samples (the same method as tm_stats.cu); windows
// where those could cancel, or whose std is near the 1e-12 cut, are recomputed with the
// reference's own two-pass arithmetic. Results equal tm_window_stats's to a few float
// ulps (bit-identical for the two-pass windows).
//
// The only scratch is the FP64 suffix-sum array, held in the file-scope device array
// below (8 MiB on every GPU that loads the library, for as long as the process runs).
#include <mutex>

#include "../../include/tremor_b200.h"
#include "tm_exact.cuh"
#include "tm_internal.cuh"

namespace tmb {
namespace noalloc {

// n + m samples at most: (windows + m) suffix sums of (x, x^2) in FP64.
constexpr uint64_t kMaxSamples = 524288;
static __device__ __align__(256) double2 g_suffix[kMaxSamples];

__device__ __forceinline__ double clean64(float v) { return v == kMissing ? 0.0 : (double)v; }

// One warp per segment [a*m, (a+1)*m) ∩ [0, n): suffix sums, read straight from raw.
__global__ void k_suffix_from_raw(const float *__restrict__ raw, uint64_t n, int m, uint64_t segments,
                                  double2 *__restrict__ suf)
{
    const uint64_t a = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (a >= segments)
        return;
    const uint64_t base = a * (uint64_t)m;
    const uint64_t end = min(base + (uint64_t)m, n);
    double cs = 0.0, cq = 0.0;
    for (int64_t hi = (int64_t)end; hi > (int64_t)base; hi -= 32)
    {
        const int64_t idx = hi - 32 + lane;
        const bool valid = idx >= (int64_t)base;
        const double v = valid ? clean64(raw[idx]) : 0.0;
        double s = v, q = v * v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const double ts = __shfl_down_sync(0xffffffffu, s, off);
            const double tq = __shfl_down_sync(0xffffffffu, q, off);
            if (lane + off < 32)
            {
                s += ts;
                q += tq;
            }
        }
        if (valid)
            suf[idx] = make_double2(s + cs, q + cq);
        cs += __shfl_sync(0xffffffffu, s, 0);
        cq += __shfl_sync(0xffffffffu, q, 0);
    }
}

__device__ __forceinline__ void finish(const float *__restrict__ raw, uint64_t j, int m, double s, double q,
                                       double r2max, float *__restrict__ mean, float *__restrict__ stddev,
                                       uint8_t *__restrict__ flags)
{
    if (raw[j] == kMissing)
    {
        mean[j] = 0.0f;
        stddev[j] = 0.0f;
        flags[j] = kFlagMissingStart;
        return;
    }
    const double mu = s / (double)m;
    const double var = q / (double)m - mu * mu;
    if (!(var > 0.0) || mu * mu > var * r2max || var < 1e-22)
    {
        float mf, sf;
        exact_stats(raw, j, m, mf, sf);
        mean[j] = mf;
        stddev[j] = sf;
        flags[j] = (uint8_t)(kFlagExact | (sf == 0.0f ? kFlagDegenerate : 0));
        return;
    }
    mean[j] = (float)mu;
    stddev[j] = (float)sqrt(var);
    flags[j] = 0;
}

// One warp per segment a: windows a*m + o, o in [0, m), from the suffix sums of segment
// a and the running prefix sums of segment a + 1.
__global__ void k_stats_from_suffix(const float *__restrict__ raw, const double2 *__restrict__ suf, uint64_t n, int m,
                                    uint64_t segments, uint64_t W, double r2max, float *__restrict__ mean,
                                    float *__restrict__ stddev, uint8_t *__restrict__ flags)
{
    const uint64_t a = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (a >= segments)
        return;
    const uint64_t base = a * (uint64_t)m;
    if (lane == 0 && base < W)
        finish(raw, base, m, suf[base].x, suf[base].y, r2max, mean, stddev, flags);
    double cs = 0.0, cq = 0.0;
    for (int p0 = 0; p0 < m - 1; p0 += 32)
    {
        const int p = p0 + lane;
        const uint64_t j = base + (uint64_t)p + 1;
        const uint64_t idx = base + (uint64_t)m + p;
        const bool in_seg = p < m - 1 && idx < n;
        const double v = in_seg ? clean64(raw[idx]) : 0.0;
        double s = v, q = v * v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const double ts = __shfl_up_sync(0xffffffffu, s, off);
            const double tq = __shfl_up_sync(0xffffffffu, q, off);
            if (lane >= off)
            {
                s += ts;
                q += tq;
            }
        }
        s += cs;
        q += cq;
        if (in_seg && j < W)
            finish(raw, j, m, suf[j].x + s, suf[j].y + q, r2max, mean, stddev, flags);
        cs = __shfl_sync(0xffffffffu, s, 31);
        cq = __shfl_sync(0xffffffffu, q, 31);
        if (base + (uint64_t)p0 + 33 >= W)
            break;
    }
}

// Device address of g_suffix on each device, resolved once per device (with that device
// current) by the first call on it and kept until the process exits: a cudaDeviceReset
// unloads the module, after which the kept address is stale.
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double2 *g_addr[kMaxDevices] = {};

} // namespace noalloc
} // namespace tmb

extern "C" int tm_window_stats_noalloc(const float *raw, uint64_t n, int m, float *mean, float *stddev,
                                       uint8_t *flags, void *stream)
{
    using namespace tmb::noalloc;
    if (raw == nullptr || mean == nullptr || stddev == nullptr || flags == nullptr || m < 1 ||
        static_cast<uint64_t>(m) > n)
        return TM_ERR_ARGUMENT;
    if (n + static_cast<uint64_t>(m) > kMaxSamples)
        return TM_ERR_TOO_LARGE; // n + m must not exceed 524288 samples (the fixed scratch)
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return TM_ERR_NO_DEVICE;
    double2 *suf = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (g_addr[dev] == nullptr)
        {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_suffix) != cudaSuccess || p == nullptr)
                return TM_ERR_CUDA;
            g_addr[dev] = static_cast<double2 *>(p);
        }
        suf = g_addr[dev];
    }
    const uint64_t W = n - static_cast<uint64_t>(m) + 1;
    const uint64_t segments = (W - 1) / static_cast<uint64_t>(m) + 1; // segments holding window starts
    const unsigned blocks = static_cast<unsigned>((segments * 32 + 255) / 256);
    const double r2max = 5e-7 / (static_cast<double>(m) * 1.1102230246251565e-16);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_suffix_from_raw<<<blocks, 256, 0, s>>>(raw, n, m, segments, suf);
    k_stats_from_suffix<<<blocks, 256, 0, s>>>(raw, suf, n, m, segments, W, r2max, mean, stddev, flags);
    return cudaGetLastError() == cudaSuccess ? TM_OK : TM_ERR_CUDA;
}
