// Answer assembly on the device, after the exact re-scoring (tm_select.cu k_rescore).
//
// The reference collects, per template, every verified window: threshold hits whose
// ED^2 <= threshold (Tremor.cpp:2008, SkipSequential.cpp:279-290) and the kNN
// candidates offered to the bound queue. Threshold post-processing sorts a template's
// hits by position (Tremor.cpp:2760-2795); the kNN answer is the canonical exclusion
// selection over the candidates in (ED^2, position) order (ZnormSearch.hpp:170-189).
// Here both happen on the device, so the host receives finished runs:
//   k_answer_keys      keeps the candidates that can be answers (threshold templates:
//                      exact ED^2 <= threshold; kNN templates: all of them) as
//                      (template << 32 | window, ED^2) pairs
//   radix sort 1       by that key: template-major, position order within a template
//   k_answer_rekey     (only when the group has kNN templates) kNN entries get the key
//                      (flag, template, ED^2 bits) and threshold entries keep
//                      (template, window); the flag, above the template bits, moves
//                      every kNN run after all threshold runs
//   radix sort 2       by the new key; the sort is stable, so equal distances stay in
//                      position order: (distance, position) order within a kNN run
//   k_answer_segments  each template's run [start, end), its windows and distances
//   k_select_knn       one warp per kNN template: the greedy exclusion selection over
//                      its run (finite distances only), up to k answers
// The sorts are CUB's device radix sort from the CUDA toolkit, over 32 + ceil(log2 T)
// (+1) key bits. Within a template no window appears twice: every (template, window)
// pair is visited by exactly one contraction tile, and the kNN re-pass lists each
// bucket once.
#include <cub/device/device_radix_sort.cuh>

#include "../../include/tremor_b200.h"
#include "tm_internal.cuh"

namespace tmb {

constexpr int kAnswerThreads = 256;
constexpr int kSelectWarps = 4;

__device__ __forceinline__ void warp_slot(bool keep, uint32_t *counter, uint32_t &slot)
{
    const unsigned ballot = __ballot_sync(0xffffffffu, keep);
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (ballot != 0u)
    {
        const int leader = __ffs(ballot) - 1;
        if (lane == leader)
            base = atomicAdd(counter, (uint32_t)__popc(ballot));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    slot = base + (uint32_t)__popc(ballot & ((1u << lane) - 1u));
}

// kept[0]: answers kept, kept[1]: of which belong to kNN templates.
__global__ void __launch_bounds__(kAnswerThreads)
    k_answer_keys(const Candidate *__restrict__ cand, const float *__restrict__ dist, uint32_t count,
                  const TemplParam *__restrict__ tp, unsigned long long *__restrict__ keys, float *__restrict__ vals,
                  uint32_t *__restrict__ kept)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool keep = false, knn = false;
    Candidate c{0u, 0u};
    float d = 0.0f;
    if (i < count)
    {
        c = cand[i];
        d = dist[i];
        knn = tp[c.templ].mode == TM_MODE_KNN;
        keep = knn || d <= tp[c.templ].thr_ed;
    }
    uint32_t slot, unused;
    warp_slot(keep, kept, slot);
    warp_slot(keep && knn, kept + 1, unused);
    if (keep)
    {
        keys[slot] = ((unsigned long long)c.templ << 32) | (unsigned long long)c.window;
        vals[slot] = d;
    }
}

__global__ void __launch_bounds__(kAnswerThreads)
    k_answer_rekey(const unsigned long long *__restrict__ keys, const float *__restrict__ vals, uint32_t count,
                   const TemplParam *__restrict__ tp, int tbits, unsigned long long *__restrict__ keys2,
                   unsigned long long *__restrict__ vals2)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const unsigned long long k = keys[i];
    const uint32_t t = (uint32_t)(k >> 32), w = (uint32_t)k;
    const float d = vals[i];
    const bool knn = tp[t].mode == TM_MODE_KNN;
    keys2[i] = knn ? (1ull << (32 + tbits)) | ((unsigned long long)t << 32) | float_key(d) : k;
    vals2[i] = ((unsigned long long)w << 32) | __float_as_uint(d);
}

// start[t], end[t] (zeroed before: templates without answers keep the empty run [0, 0)),
// and the run's windows and distances. PACKED: values are (window << 32 | ED^2 bits);
// otherwise the window is the key's low half and the values are the distances.
template <bool PACKED>
__global__ void __launch_bounds__(kAnswerThreads)
    k_answer_segments(const unsigned long long *__restrict__ keys, const void *__restrict__ vals, uint32_t count,
                      uint32_t tmask, uint32_t *__restrict__ start, uint32_t *__restrict__ end,
                      uint32_t *__restrict__ window, float *__restrict__ dist)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const uint32_t t = (uint32_t)(keys[i] >> 32) & tmask;
    if (PACKED)
    {
        const unsigned long long v = static_cast<const unsigned long long *>(vals)[i];
        window[i] = (uint32_t)(v >> 32);
        dist[i] = __uint_as_float((uint32_t)v);
    }
    else
    {
        window[i] = (uint32_t)keys[i];
        dist[i] = static_cast<const float *>(vals)[i];
    }
    if (i == 0 || ((uint32_t)(keys[i - 1] >> 32) & tmask) != t)
        start[t] = i;
    if (i + 1 == count || ((uint32_t)(keys[i + 1] >> 32) & tmask) != t)
        end[t] = i + 1;
}

// Greedy exclusion selection of one kNN template per warp over its run in (distance,
// position) order: a candidate is kept when no kept window lies closer than merge
// (|gap| < merge), until k are kept (ZnormSearch.hpp:170-189). Only finite distances
// take part; the run's FLT_MAX entries, at its end, are left to the host, which needs
// them only when the reference's queue would not have filled. Lanes take 32 candidates
// at a time; the survivors of the kept-set check are accepted in lane order, each one
// removing the later survivors within merge of it. out_n[slot] = answers kept.
__global__ void __launch_bounds__(kSelectWarps * 32)
    k_select_knn(const int *__restrict__ slots, int nk, const TemplParam *__restrict__ tp,
                 const uint32_t *__restrict__ start, const uint32_t *__restrict__ end,
                 const uint32_t *__restrict__ window, const float *__restrict__ dist, int kcap,
                 uint32_t *__restrict__ out_n, uint32_t *__restrict__ out_win, float *__restrict__ out_dist)
{
    extern __shared__ uint32_t kept_win[]; // kSelectWarps x kcap
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = blockIdx.x * kSelectWarps + warp;
    if (slot >= nk)
        return; // whole warp
    const int t = slots[slot];
    const int k = min(tp[t].k, kcap);
    const uint32_t merge = (uint32_t)max(tp[t].merge, 0);
    const uint32_t a = start[t], b = end[t];
    uint32_t *kw = kept_win + warp * kcap;
    uint32_t *ow = out_win + (size_t)slot * kcap;
    float *od = out_dist + (size_t)slot * kcap;
    int n = 0;
    for (uint32_t base = a; base < b && n < k; base += 32)
    {
        const uint32_t i = base + lane;
        const bool valid = i < b;
        const uint32_t w = valid ? window[i] : 0u;
        const float d = valid ? dist[i] : 0.0f;
        bool pass = valid && d < kFltMax;
        if (merge > 0 && pass)
            for (int j = 0; j < n; j++)
            {
                const uint32_t kj = kw[j];
                if ((w > kj ? w - kj : kj - w) < merge)
                {
                    pass = false;
                    break;
                }
            }
        const bool last = __any_sync(0xffffffffu, valid && !(d < kFltMax));
        unsigned pb = __ballot_sync(0xffffffffu, pass);
        while (pb != 0u && n < k)
        {
            const int leader = __ffs(pb) - 1;
            const uint32_t lw = __shfl_sync(0xffffffffu, w, leader);
            const float ld = __shfl_sync(0xffffffffu, d, leader);
            if (lane == 0)
            {
                kw[n] = lw;
                ow[n] = lw;
                od[n] = ld;
            }
            n++;
            if (lane == leader || (pass && (w > lw ? w - lw : lw - w) < merge))
                pass = false;
            pb = __ballot_sync(0xffffffffu, pass);
        }
        __syncwarp();
        if (last)
            break;
    }
    if (lane == 0)
        out_n[slot] = (uint32_t)n;
}

// Key bits for T templates: the window's 32 and enough for the template index.
int answer_template_bits(int T)
{
    int b = 0;
    while (b < 30 && (1u << b) < (uint32_t)T)
        b++;
    return b;
}

cudaError_t launch_answer_keys(const Candidate *cand, const float *dist, uint32_t count, const TemplParam *tp,
                               unsigned long long *keys, float *vals, uint32_t *kept, cudaStream_t s)
{
    if (count > 0)
        k_answer_keys<<<(count + kAnswerThreads - 1) / kAnswerThreads, kAnswerThreads, 0, s>>>(cand, dist, count, tp,
                                                                                              keys, vals, kept);
    return cudaGetLastError();
}

// Scratch bytes both sorts need for `count` pairs (a size query: nothing is launched).
size_t answer_sort_scratch(uint32_t count, int T)
{
    const int tb = answer_template_bits(T);
    size_t b1 = 0, b2 = 0;
    cub::DoubleBuffer<unsigned long long> k(nullptr, nullptr), v64(nullptr, nullptr);
    cub::DoubleBuffer<float> v32(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairs(nullptr, b1, k, v32, count, 0, 32 + tb);
    cub::DeviceRadixSort::SortPairs(nullptr, b2, k, v64, count, 0, 33 + tb);
    return b1 > b2 ? b1 : b2;
}

// The answer order of the `count` kept pairs in (keys[0], vals32[0]); knn_count of them
// belong to kNN templates. Leaves each template's run in start/end, its windows in
// `window` and distances in `dist` (count entries each; threshold runs first).
cudaError_t launch_answer_order(unsigned long long *const keys[2], float *const vals32[2],
                                unsigned long long *const vals64[2], uint32_t count, uint32_t knn_count,
                                const TemplParam *tp, int T, void *scratch, size_t scratch_bytes, uint32_t *start,
                                uint32_t *end, uint32_t *window, float *dist, cudaStream_t s)
{
    if (count == 0)
        return cudaSuccess;
    const int tb = answer_template_bits(T);
    const uint32_t tmask = (1u << tb) - 1u;
    const unsigned grid = (count + kAnswerThreads - 1) / kAnswerThreads;
    cub::DoubleBuffer<unsigned long long> k(keys[0], keys[1]);
    cub::DoubleBuffer<float> v(vals32[0], vals32[1]);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(scratch, scratch_bytes, k, v, count, 0, 32 + tb, s);
    if (e != cudaSuccess)
        return e;
    if (k.selector != v.selector)
        return cudaErrorUnknown;
    if (knn_count == 0)
    {
        k_answer_segments<false><<<grid, kAnswerThreads, 0, s>>>(k.Current(), v.Current(), count, ~0u, start,
                                                                 end, window, dist);
        return cudaGetLastError();
    }
    unsigned long long *k2a = k.Alternate(), *k2b = k.Current();
    k_answer_rekey<<<grid, kAnswerThreads, 0, s>>>(k.Current(), v.Current(), count, tp, tb, k2a, vals64[0]);
    cub::DoubleBuffer<unsigned long long> k2(k2a, k2b), v2(vals64[0], vals64[1]);
    e = cub::DeviceRadixSort::SortPairs(scratch, scratch_bytes, k2, v2, count, 0, 33 + tb, s);
    if (e != cudaSuccess)
        return e;
    if (k2.selector != v2.selector)
        return cudaErrorUnknown;
    k_answer_segments<true><<<grid, kAnswerThreads, 0, s>>>(k2.Current(), v2.Current(), count, tmask, start, end,
                                                            window, dist);
    return cudaGetLastError();
}

cudaError_t launch_select_knn(const int *slots, int nk, const TemplParam *tp, const uint32_t *start,
                              const uint32_t *end, const uint32_t *window, const float *dist, int kcap,
                              uint32_t *out_n, uint32_t *out_win, float *out_dist, cudaStream_t s)
{
    if (nk > 0)
        k_select_knn<<<(nk + kSelectWarps - 1) / kSelectWarps, kSelectWarps * 32,
                       sizeof(uint32_t) * kSelectWarps * kcap, s>>>(slots, nk, tp, start, end, window, dist, kcap,
                                                                    out_n, out_win, out_dist);
    return cudaGetLastError();
}

} // namespace tmb
