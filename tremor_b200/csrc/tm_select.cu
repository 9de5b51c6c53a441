// kNN bound selection, bucket re-pass and exact re-scoring.
//
// Why a bound from bucket minima is valid. The reference's kNN answer is the
// canonical exclusion selection (ZnormSearch.hpp:170-189) over every searched window
// ordered by (FP32 distance, position); its bound queue (2k-1 pairwise separated
// entries with a merge offset, k without, SkipSequential.cpp:378-379) only prunes.
// If 2k-1 windows pairwise at least merge_offset apart all have distance <= T, every
// one of the k answers has distance <= T: each kept answer excludes at most two of
// them (one on each side), so after fewer than k picks one of them is still free.
// Minima over buckets of >= merge_offset windows taken from every other bucket are
// pairwise separated, so with u = d + E >= reference distance,
//     T = min over the two parities of the (2k-1)-th smallest bucket minimum of u
// is such a bound (for merge_offset 0: the k-th smallest over all buckets). Every
// window with reference distance <= T has d - E <= T, so re-scoring the windows of
// the buckets whose minimum of d - E is <= T, and keeping those with d - E <= T,
// yields a candidate set that contains every window the canonical selection can
// pick before it has k answers.
#include "tm_epilogue.cuh"
#include "tm_exact.cuh"
#include "tm_internal.cuh"
#include "tm_prefix.cuh"

namespace tmb {

// r-th smallest (1-based) of `count` keys produced by value(i), by 8-bit radix select
// over the whole block; returns kEmptyKey when count < r.
template <class F> __device__ uint32_t block_select(F value, uint32_t count, uint32_t r)
{
    __shared__ uint32_t hist[256];
    __shared__ uint32_t s_prefix, s_r;
    if (count < r)
        return kEmptyKey;
    uint32_t prefix = 0, mask = 0;
    if (threadIdx.x == 0)
        s_r = r;
    for (int shift = 24; shift >= 0; shift -= 8)
    {
        for (int i = threadIdx.x; i < 256; i += blockDim.x)
            hist[i] = 0;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < count; i += blockDim.x)
        {
            const uint32_t key = value(i);
            if ((key & mask) == prefix)
                atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            uint32_t rr = s_r, digit = 0;
            for (; digit < 255; digit++)
            {
                if (hist[digit] >= rr)
                    break;
                rr -= hist[digit];
            }
            s_r = rr;
            s_prefix = prefix | (digit << shift);
        }
        __syncthreads();
        prefix = s_prefix;
        mask |= 255u << shift;
        __syncthreads();
    }
    return prefix;
}

// One block per kNN template slot: tkey[t] = key of the bound T (kEmptyKey: +inf).
__global__ void k_bucket_select(const uint32_t *__restrict__ bmin_u, uint32_t nb, const TemplParam *__restrict__ tp,
                                const int *__restrict__ knn_slots, uint32_t *__restrict__ tkey)
{
    const int t = knn_slots[blockIdx.x];
    const TemplParam p = tp[t];
    const uint32_t *u = bmin_u + (size_t)t * nb;
    uint32_t result;
    if (p.merge <= 0)
    {
        result = block_select([&](uint32_t i) { return u[i]; }, nb, (uint32_t)p.k);
    }
    else
    {
        const uint32_t sb = (uint32_t)((p.merge + kBucket - 1) / kBucket); // buckets per super-bucket
        const uint32_t nsb = (nb + sb - 1) / sb;
        result = kEmptyKey;
        for (uint32_t parity = 0; parity < 2; parity++)
        {
            const uint32_t cnt = nsb > parity ? (nsb - parity + 1) / 2 : 0;
            const uint32_t r = block_select(
                [&](uint32_t i) {
                    const uint32_t s = 2 * i + parity;
                    uint32_t best = kEmptyKey;
                    for (uint32_t b = s * sb; b < min((s + 1) * sb, nb); b++)
                        best = min(best, u[b]);
                    return best;
                },
                cnt, (uint32_t)(2 * p.k - 1));
            result = min(result, r);
        }
    }
    if (threadIdx.x == 0)
        tkey[t] = result;
}

// (template slot, bucket) pairs whose minimum of d - E is within the bound.
__global__ void k_list_buckets(const uint32_t *__restrict__ bmin_l, uint32_t nb, const int *__restrict__ knn_slots,
                               int nk, const uint32_t *__restrict__ tkey, uint2 *__restrict__ list,
                               uint32_t *__restrict__ list_count, uint32_t cap)
{
    const uint64_t total = (uint64_t)nk * nb;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x)
    {
        const int t = knn_slots[i / nb];
        const uint32_t b = (uint32_t)(i % nb);
        const uint32_t l = bmin_l[(size_t)t * nb + b];
        if (l != kEmptyKey && l <= tkey[t])
        {
            const uint32_t at = atomicAdd(list_count, 1u);
            if (at < cap)
                list[at] = make_uint2((uint32_t)t, b);
        }
    }
}

constexpr int B_THREADS = 256, B_KC = 512;

// FP32 re-pass over one listed bucket of one template: every window with d - E <= T.
__global__ void __launch_bounds__(B_THREADS) k_passb(const uint2 *__restrict__ list, const float *__restrict__ x,
                                                     const float *__restrict__ q, const TemplParam *__restrict__ tp,
                                                     const float *__restrict__ mean, const float *__restrict__ inv,
                                                     const uint32_t *__restrict__ tkey, uint64_t w0, uint32_t W,
                                                     Candidate *cand, uint32_t *cand_count, uint32_t cand_cap)
{
    __shared__ __align__(16) float xs[kBucket + B_KC + 16];
    __shared__ __align__(16) float qs[B_KC];
    const uint2 item = list[blockIdx.x];
    const uint32_t t = item.x;
    const TemplParam p = tp[t];
    const uint32_t tk = tkey[t];
    const float T = tk == kEmptyKey ? inf_f() : key_float(tk);
    const uint32_t jb = item.y * kBucket;
    const float shift = mean[min(jb + kBucket / 2, W - 1)];
    const float *xg = x + w0 + jb;
    const float *qg = q + p.q_offset;
    const int m_pad = (p.m + 63) & ~63;
    const int tid = threadIdx.x, lane = tid & 31;
    float acc[8];
#pragma unroll
    for (int w = 0; w < 8; w++)
        acc[w] = 0.0f;
    for (int k0 = 0; k0 < m_pad; k0 += B_KC)
    {
        const int kc = min(B_KC, m_pad - k0);
        for (int i = tid; i < kBucket + kc; i += B_THREADS)
            xs[i] = xg[k0 + i] - shift;
        for (int i = tid; i < kc; i += B_THREADS)
            qs[i] = qg[k0 + i];
        __syncthreads();
        const float *xw = xs + 8 * tid;
        for (int kk = 0; kk < kc; kk += 4)
        {
            const float4 xa = *reinterpret_cast<const float4 *>(xw + kk);
            const float4 xb = *reinterpret_cast<const float4 *>(xw + kk + 4);
            const float4 xc = *reinterpret_cast<const float4 *>(xw + kk + 8);
            const float4 qv = *reinterpret_cast<const float4 *>(qs + kk);
            const float xr[12] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w, xc.x, xc.y, xc.z, xc.w};
#pragma unroll
            for (int w = 0; w < 8; w++)
            {
                acc[w] = fmaf(xr[w + 0], qv.x, acc[w]);
                acc[w] = fmaf(xr[w + 1], qv.y, acc[w]);
                acc[w] = fmaf(xr[w + 2], qv.z, acc[w]);
                acc[w] = fmaf(xr[w + 3], qv.w, acc[w]);
            }
        }
        __syncthreads();
    }
    const uint32_t j0 = jb + 8 * tid;
    uint32_t mask = 0;
#pragma unroll
    for (int w = 0; w < 8; w++)
    {
        const uint32_t j = j0 + w;
        if (j >= W)
            continue;
        const float iv = inv[j];
        if (iv == 0.0f)
            continue;
        float d, e;
        fast_distance(p, p.a1_fp32, acc[w], mean[j], iv, shift, d, e);
        if (d - e <= T)
            mask |= 1u << w;
    }
    emit_candidates(mask, lane, t, j0, cand, cand_count, cand_cap);
}

// k_passb for tiles of several template lengths: statistics from the prefix sums, and
// windows whose statistics are not trustworthy are always emitted (re-scored exactly).
__global__ void __launch_bounds__(B_THREADS) k_passb_mixed(const uint2 *__restrict__ list, const float *__restrict__ x,
                                                           const float *__restrict__ raw, const PrefixView pv,
                                                           const uint16_t *__restrict__ run,
                                                           const float *__restrict__ q,
                                                           const TemplParam *__restrict__ tp,
                                                           const uint32_t *__restrict__ tkey, uint64_t w0,
                                                           Candidate *cand, uint32_t *cand_count, uint32_t cand_cap)
{
    __shared__ __align__(16) float xs[kBucket + B_KC + 16];
    __shared__ __align__(16) float qs[B_KC];
    const uint2 item = list[blockIdx.x];
    const uint32_t t = item.x;
    const TemplParam p = tp[t];
    const uint32_t tk = tkey[t];
    const float T = tk == kEmptyKey ? inf_f() : key_float(tk);
    const uint32_t jb = item.y * kBucket;
    const float shift = x[w0 + min(jb + kBucket / 2, p.wcount - 1)];
    const float *xg = x + w0 + jb;
    const float *qg = q + p.q_offset;
    const int m_pad = (p.m + 63) & ~63;
    const int tid = threadIdx.x, lane = tid & 31;
    float acc[8];
#pragma unroll
    for (int w = 0; w < 8; w++)
        acc[w] = 0.0f;
    for (int k0 = 0; k0 < m_pad; k0 += B_KC)
    {
        const int kc = min(B_KC, m_pad - k0);
        for (int i = tid; i < kBucket + kc; i += B_THREADS)
            xs[i] = xg[k0 + i] - shift;
        for (int i = tid; i < kc; i += B_THREADS)
            qs[i] = qg[k0 + i];
        __syncthreads();
        const float *xw = xs + 8 * tid;
        for (int kk = 0; kk < kc; kk += 4)
        {
            const float4 xa = *reinterpret_cast<const float4 *>(xw + kk);
            const float4 xb = *reinterpret_cast<const float4 *>(xw + kk + 4);
            const float4 xc = *reinterpret_cast<const float4 *>(xw + kk + 8);
            const float4 qv = *reinterpret_cast<const float4 *>(qs + kk);
            const float xr[12] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w, xc.x, xc.y, xc.z, xc.w};
#pragma unroll
            for (int w = 0; w < 8; w++)
            {
                acc[w] = fmaf(xr[w + 0], qv.x, acc[w]);
                acc[w] = fmaf(xr[w + 1], qv.y, acc[w]);
                acc[w] = fmaf(xr[w + 2], qv.z, acc[w]);
                acc[w] = fmaf(xr[w + 3], qv.w, acc[w]);
            }
        }
        __syncthreads();
    }
    const uint32_t j0 = jb + 8 * tid;
    uint32_t mask = 0;
#pragma unroll
    for (int w = 0; w < 8; w++)
    {
        const uint32_t j = j0 + w;
        if (j >= p.wcount || raw[w0 + j] == kMissing || run[w0 + j] >= p.m)
            continue;
        WindowStats ws;
        if (window_prefix_stats(pv, pv.Q[w0 + j], pv.Q[w0 + j + p.m], w0 + j, p.m, p.inv_m, ws) != 0)
        {
            mask |= 1u << w;
            continue;
        }
        float d, e;
        fast_distance_mixed(p, p.a1_fp32, acc[w], ws.mu, ws.iv, shift, stats_error(ws, p.m, p.qs, p.s1), d, e);
        if (d - e <= T)
            mask |= 1u << w;
    }
    emit_candidates(mask, lane, t, j0, cand, cand_count, cand_cap);
}

// Exact (reference-arithmetic) distance of every candidate.
__global__ void k_rescore(const Candidate *__restrict__ cand, uint32_t count, const TemplParam *__restrict__ tp,
                          const float *__restrict__ q, const int *__restrict__ order, const float *__restrict__ raw,
                          uint64_t w0, float *__restrict__ dist)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const Candidate c = cand[i];
    const TemplParam p = tp[c.templ];
    const uint64_t g = w0 + c.window;
    float mean_f, std_f;
    exact_stats(raw, g, p.m, mean_f, std_f);
    dist[i] = replica_distance(q + p.q_offset, order + p.order_offset, raw, g, p.m, mean_f, std_f);
}

// ---- launchers --------------------------------------------------------------------

cudaError_t launch_bucket_select(const uint32_t *bmin_u, uint32_t nb, const TemplParam *tp, const int *knn_slots,
                                 int nk, uint32_t *tkey, cudaStream_t s)
{
    if (nk > 0)
        k_bucket_select<<<nk, 1024, 0, s>>>(bmin_u, nb, tp, knn_slots, tkey);
    return cudaGetLastError();
}

cudaError_t launch_list_buckets(const uint32_t *bmin_l, uint32_t nb, const int *knn_slots, int nk,
                                const uint32_t *tkey, uint2 *list, uint32_t *list_count, uint32_t cap, cudaStream_t s)
{
    if (nk > 0)
        k_list_buckets<<<1184, 256, 0, s>>>(bmin_l, nb, knn_slots, nk, tkey, list, list_count, cap);
    return cudaGetLastError();
}

cudaError_t launch_passb(const uint2 *list, uint32_t items, const float *x, const float *q, const TemplParam *tp,
                         const float *mean, const float *inv, const uint32_t *tkey, uint64_t w0, uint32_t W,
                         Candidate *cand, uint32_t *cand_count, uint32_t cand_cap, cudaStream_t s)
{
    if (items > 0)
        k_passb<<<items, B_THREADS, 0, s>>>(list, x, q, tp, mean, inv, tkey, w0, W, cand, cand_count, cand_cap);
    return cudaGetLastError();
}

cudaError_t launch_passb_mixed(const uint2 *list, uint32_t items, const float *x, const float *raw, const double2 *P,
                               const double2 *PT, const double *PC, const uint16_t *run, const float *q,
                               const TemplParam *tp,
                               const uint32_t *tkey, uint64_t w0, Candidate *cand, uint32_t *cand_count,
                               uint32_t cand_cap, cudaStream_t s)
{
    if (items > 0)
        k_passb_mixed<<<items, B_THREADS, 0, s>>>(list, x, raw, PrefixView{P, PT, PC}, run, q, tp, tkey, w0, cand, cand_count,
                                                  cand_cap);
    return cudaGetLastError();
}

cudaError_t launch_rescore(const Candidate *cand, uint32_t count, const TemplParam *tp, const float *q,
                           const int *order, const float *raw, uint64_t w0, float *dist, cudaStream_t s)
{
    if (count > 0)
        k_rescore<<<(count + 127) / 128, 128, 0, s>>>(cand, count, tp, q, order, raw, w0, dist);
    return cudaGetLastError();
}

} // namespace tmb
