// C ABI of tremor_b200 (include/tremor_b200.h): context, window statistics, batched
// searches, results. One search of a group of same-length templates runs:
//
//   1. host: z-normalise each template (bit-identical to the reference), block order,
//      epilogue constants;                                        (tm_host.cpp)
//   2. device: contraction kernel with fused epilogue: threshold candidates and
//      per-bucket minima for kNN;                (tm_scan_fp32.cu / tm_scan_umma.cu)
//   3. device, kNN only: bound from bucket minima, list of buckets within it, FP32
//      re-pass of those buckets emitting the kNN candidates;        (tm_select.cu)
//   4. device: every candidate re-scored with the reference's exact arithmetic;
//   5. host: canonical exclusion selection / threshold merge on the exact distances.
#include <algorithm>
#include <functional>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/tremor_b200.h"
#include "tm_epilogue.cuh"
#include "tm_host.h"
#include "tm_internal.cuh"
#include "tm_prefix.cuh"
#include "tm_fft.cuh"

#include <cufft.h>

namespace tmb {
cudaError_t launch_clean(const float *raw, float *clean, uint64_t n, uint64_t n_total, cudaStream_t s);
cudaError_t launch_window_stats(const float *clean, const float *raw, uint64_t n, int m, uint64_t w0, uint64_t W,
                                double2 *suf, float *mean, float *inv, uint8_t *flags, cudaStream_t s);
cudaError_t launch_reference_stats(const float *raw, int m, uint64_t w0, uint64_t count, float *mean, float *stddev,
                                   cudaStream_t s);
cudaError_t launch_scan_fp32(const ScanArgs &a, cudaStream_t s);
cudaError_t launch_scan_umma(const ScanArgs &a, cudaStream_t s);
cudaError_t launch_scan_wm(const ScanArgs &a, cudaStream_t s);
bool umma_supported(int m, int T, uint64_t W);
cudaError_t launch_bucket_select(const uint32_t *bmin_u, uint32_t nb, const TemplParam *tp, const int *knn_slots,
                                 int nk, uint32_t *tkey, cudaStream_t s);
cudaError_t launch_list_buckets(const uint32_t *bmin_l, uint32_t nb, const int *knn_slots, int nk,
                                const uint32_t *tkey, uint2 *list, uint32_t *list_count, uint32_t cap, cudaStream_t s);
cudaError_t launch_passb(const uint2 *list, uint32_t items, const float *x, const float *q, const TemplParam *tp,
                         const float *mean, const float *inv, const uint32_t *tkey, uint64_t w0, uint32_t W,
                         Candidate *cand, uint32_t *cand_count, uint32_t cand_cap, cudaStream_t s);
cudaError_t launch_rescore(const Candidate *cand, uint32_t count, const TemplParam *tp, const float *q,
                           const int *order, const float *raw, uint64_t w0, float *dist, cudaStream_t s);
uint32_t prefix_chunks(uint64_t n);
cudaError_t launch_prefix_totals(const float *clean, uint64_t n, const double *centres, double2 *totals,
                                 cudaStream_t s);
cudaError_t launch_prefix_sums(const float *clean, uint64_t n, const double *centres, double2 *totals,
                               double2 *block_totals, double2 *Q, cudaStream_t s);
cudaError_t launch_runs(const float *clean, uint64_t n, uint16_t *run, uint16_t *run_tmp, cudaStream_t s);
cudaError_t launch_passb_mixed(const uint2 *list, uint32_t items, const float *x, const float *raw, const double2 *P,
                               const double2 *PT, const double *PC, const uint16_t *run, const float *q,
                               const TemplParam *tp, const uint32_t *tkey, uint64_t w0, Candidate *cand,
                               uint32_t *cand_count, uint32_t cand_cap, cudaStream_t s);
cudaError_t launch_answer_keys(const Candidate *cand, const float *dist, uint32_t count, const TemplParam *tp,
                               unsigned long long *keys, float *vals, uint32_t *kept, cudaStream_t s);
size_t answer_sort_scratch(uint32_t count, int T);
cudaError_t launch_answer_order(unsigned long long *const keys[2], float *const vals32[2],
                                unsigned long long *const vals64[2], uint32_t count, uint32_t knn_count,
                                const TemplParam *tp, int T, void *scratch, size_t scratch_bytes, uint32_t *start,
                                uint32_t *end, uint32_t *window, float *dist, cudaStream_t s);
cudaError_t launch_select_knn(const int *slots, int nk, const TemplParam *tp, const uint32_t *start,
                              const uint32_t *end, const uint32_t *window, const float *dist, int kcap,
                              uint32_t *out_n, uint32_t *out_win, float *out_dist, cudaStream_t s);
} // namespace tmb

using tmb::Candidate;
using tmb::TemplParam;
using tm_host::Hit;

namespace {

struct Failure
{
    int code;
    std::string what;
};

#define TM_CUDA(call)                                                                                             \
    do                                                                                                            \
    {                                                                                                             \
        cudaError_t e_ = (call);                                                                                  \
        if (e_ != cudaSuccess)                                                                                    \
            throw Failure{e_ == cudaErrorMemoryAllocation ? TM_ERR_NO_MEMORY : TM_ERR_CUDA,                      \
                          std::string(#call) + ": " + cudaGetErrorString(e_)};                                    \
    } while (0)

// Grow-only device buffer.
struct DevBuf
{
    void *p = nullptr;
    size_t bytes = 0;
    void reserve(size_t need)
    {
        if (need <= bytes)
            return;
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
        size_t b = std::max<size_t>(need, 256);
        TM_CUDA(cudaMalloc(&p, b));
        bytes = b;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
    void release()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

// Grow-only pinned host buffer.
struct HostBuf
{
    void *p = nullptr;
    size_t bytes = 0;
    void reserve(size_t need)
    {
        if (need <= bytes)
            return;
        if (p)
            cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        TM_CUDA(cudaMallocHost(&p, std::max<size_t>(need, 256)));
        bytes = std::max<size_t>(need, 256);
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
    void release()
    {
        if (p)
            cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
    }
};

struct LengthStats
{
    int m = 0;
    uint64_t w0 = 0, W = 0;
    DevBuf mean, inv, flags;
    uint64_t last_use = 0;
    size_t bytes() const { return mean.bytes + inv.bytes + flags.bytes; }
};

// BF16 bits of a float, round to nearest even (finite inputs).
inline uint16_t bf16_bits(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return static_cast<uint16_t>(u >> 16);
}
inline float bf16_value(uint16_t h)
{
    const uint32_t u = static_cast<uint32_t>(h) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

constexpr double kU = 5.9604644775390625e-08;   // 2^-24
constexpr double kE64 = 1.1102230246251565e-16; // 2^-53

} // namespace

// Pinned host memory holding the answers of one group; results keep it alive (shared)
// while the context hands its pool's idle blocks to later searches.
struct PinnedBlock
{
    void *p = nullptr;
    size_t bytes = 0;
    explicit PinnedBlock(size_t b)
    {
        TM_CUDA(cudaMallocHost(&p, b));
        bytes = b;
    }
    PinnedBlock(const PinnedBlock &) = delete;
    PinnedBlock &operator=(const PinnedBlock &) = delete;
    ~PinnedBlock()
    {
        if (p)
            cudaFreeHost(p);
    }
};

// Answers of one request: hits selected on the host (kNN, empty searches), or a run of
// a pinned block (threshold requests: window numbers relative to w0 and ED^2, in
// position order, as the device sorted them).
struct Answer
{
    std::vector<Hit> hits;
    const uint32_t *win = nullptr;
    const float *dist = nullptr;
    uint64_t w0 = 0, count = 0;
    bool run = false;
    uint64_t size() const { return run ? count : hits.size(); }
    Hit at(uint64_t i) const { return run ? Hit{w0 + win[i], dist[i]} : hits[i]; }
    void set_hits(std::vector<Hit> h)
    {
        hits = std::move(h);
        run = false;
    }
};

struct tm_result
{
    std::vector<Answer> answers;
    std::vector<std::shared_ptr<PinnedBlock>> blocks;
};

// The device state of one search in flight: a stream, its events, the search's scratch
// buffers and pinned staging, and its counters. The synchronous calls use the context's
// main lane; each serving worker owns one more, so searches on different lanes overlap
// (one's host work and copies with another's kernels).
struct Lane
{
    cudaStream_t stream = nullptr;
    DevBuf tkey, bmin_u, bmin_l, list, counters, cand, dist;
    // answer assembly: sort keys and values (double buffers), sort scratch, runs
    DevBuf akeys, avals, avals64, sort_tmp, segs;
    std::vector<std::shared_ptr<PinnedBlock>> pool;
    HostBuf h_split, h_q, h_order, h_slots, h_counters;
    uint32_t cand_cap = 1u << 22, list_cap = 1u << 20;
    // FFT branch: plans (one template; a batch of pieces) and buffers, created on first use
    cufftHandle fft_plan1 = 0, fft_planB = 0;
    bool fft_plans = false;
    DevBuf fft_y, fft_Y, fft_Z, fft_out;
    // instrumentation
    bool profile = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr, ev4 = nullptr;
    std::string kname;
    // milliseconds per phase: contraction, kNN bound + bucket list + re-pass, exact
    // re-scoring, answer sort, copy to the host, answer selection on the host
    double phase_ms[TM_PHASES] = {};
    int64_t prof_launches = 0, all_launches = 0;
    double prof_ms = 0.0, prof_flops = 0.0;
    uint64_t last_candidates = 0;
    uint64_t d2h_bytes = 0;

    void open()
    {
        TM_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        for (cudaEvent_t *e : {&ev0, &ev1, &ev2, &ev3, &ev4})
            TM_CUDA(cudaEventCreate(e));
    }
    void close()
    {
        if (stream)
            cudaStreamSynchronize(stream);
        if (fft_plans)
        {
            cufftDestroy(fft_plan1);
            cufftDestroy(fft_planB);
            fft_plans = false;
        }
        for (DevBuf *b : {&tkey, &bmin_u, &bmin_l, &list, &counters, &cand, &dist, &akeys, &avals, &avals64, &sort_tmp,
                          &segs, &fft_y, &fft_Y, &fft_Z, &fft_out})
            b->release();
        for (HostBuf *b : {&h_split, &h_q, &h_order, &h_slots, &h_counters})
            b->release();
        pool.clear(); // blocks still held by results are freed with the last of them
        for (cudaEvent_t *e : {&ev0, &ev1, &ev2, &ev3, &ev4})
            if (*e)
            {
                cudaEventDestroy(*e);
                *e = nullptr;
            }
        if (stream)
            cudaStreamDestroy(stream);
        stream = nullptr;
    }
};

struct Server;

struct tm_ctx
{
    int device = 0;
    uint64_t n = 0;
    DevBuf raw, clean;
    uint64_t range_first = 0, range_count = UINT64_MAX;
    int kernel = TM_KERNEL_AUTO;
    int tiles = TM_TILES_AUTO;
    // tiling cost model: kernel milliseconds for 128 templates x 2^25 windows, per group kind
    // (one length / several), shape (row tiles; column tiles of 128, 64, 32) and K (256,
    // 1024, 4096, 16384). Defaults: a B200 measurement; tm_autotune re-measures.
    double tile_ms[2][4][4] = {{{17.5, 19.3, 68.8, 272.5},
                                {29.9, 32.1, 90.9, 346.8},
                                {31.8, 43.5, 157.4, 580.8},
                                {36.7, 84.3, 308.9, 1129.8}},
                               {{31.9, 35.9, 67.5, 261.8},
                                {65.1, 70.5, 100.6, 351.7},
                                {69.0, 78.3, 159.3, 580.5},
                                {75.7, 92.5, 310.2, 1135.9}}};
    std::map<int, std::unique_ptr<LengthStats>> lengths;
    uint64_t use_clock = 0;
    DevBuf suf; // window-statistics scratch (per-length statistics)
    // length-independent statistics (mixed-length batches): block-local FP64 prefix sums,
    // their block totals and centres, constant runs
    DevBuf prefix, ptot, pcen, run;
    bool prefix_ready = false;
    // FFT branch: spectra of the record's pieces, their shifts and norms (built on first use)
    DevBuf fft_X, fft_shift, fft_norm;
    uint32_t fft_P = 0;
    bool fft_ready = false;
    std::mutex fft_mu;
    double fft_ms = 1.4; // model: ms per template per 2^25 samples (B200; tm_autotune measures it)
    std::string err;
    Lane main;                      // the synchronous calls' lane
    std::unique_ptr<Server> server; // serving engine, while started
};

namespace {

int fail(tm_ctx *ctx, const Failure &f)
{
    if (ctx)
        ctx->err = f.what;
    return f.code;
}

template <class F> int guarded(tm_ctx *ctx, F body)
{
    try
    {
        body();
        if (ctx)
            ctx->err.clear();
        return TM_OK;
    }
    catch (const Failure &f)
    {
        return fail(ctx, f);
    }
    catch (const std::bad_alloc &)
    {
        return fail(ctx, Failure{TM_ERR_NO_MEMORY, "host allocation failed"});
    }
}

void count_launch(Lane &L, int k = 1) { L.all_launches += k; }

LengthStats &ensure_length(tm_ctx *ctx, Lane &L, int m)
{
    auto it = ctx->lengths.find(m);
    if (it != ctx->lengths.end())
    {
        it->second->last_use = ++ctx->use_clock;
        return *it->second;
    }
    const uint64_t total = ctx->n - static_cast<uint64_t>(m) + 1; // windows of the whole waveform
    const uint64_t w0 = std::min(ctx->range_first, total);
    const uint64_t W = std::min(ctx->range_count, total - w0);
    // keep the resident statistics under half of the free memory: evict least recently used
    size_t free_b = 0, total_b = 0;
    TM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t need = W * 9 + 4096;
    while (!ctx->lengths.empty() && need * 2 > free_b)
    {
        auto victim = ctx->lengths.begin();
        for (auto jt = ctx->lengths.begin(); jt != ctx->lengths.end(); ++jt)
            if (jt->second->last_use < victim->second->last_use)
                victim = jt;
        free_b += victim->second->bytes();
        victim->second->mean.release();
        victim->second->inv.release();
        victim->second->flags.release();
        ctx->lengths.erase(victim);
    }
    auto ls = std::make_unique<LengthStats>();
    ls->m = m;
    ls->w0 = w0;
    ls->W = W;
    if (W > 0)
    {
        ls->mean.reserve(W * sizeof(float) + 64);
        ls->inv.reserve(W * sizeof(float) + 64);
        ls->flags.reserve(W + 64);
        const uint64_t a_count = (w0 + W - 1) / m - w0 / m + 1;
        ctx->suf.reserve(a_count * static_cast<uint64_t>(m) * sizeof(double2));
        TM_CUDA(tmb::launch_window_stats(ctx->clean.as<float>(), ctx->raw.as<float>(), ctx->n, m, w0, W,
                                        ctx->suf.as<double2>(), ls->mean.as<float>(), ls->inv.as<float>(),
                                        ls->flags.as<uint8_t>(), L.stream));
        count_launch(L, 3);
    }
    ls->last_use = ++ctx->use_clock;
    LengthStats &ref = *ls;
    ctx->lengths[m] = std::move(ls);
    return ref;
}

// Epilogue constants of one template (error-bound terms of fast_distance).
void fill_param(TemplParam &p, int m, double q2, double s1, double gamma_main, double gamma_fp32)
{
    const double qn = std::sqrt(q2), qs = qn * std::sqrt(static_cast<double>(m));
    const double md = static_cast<double>(m);
    const double safety = 1.25;
    p.s1 = static_cast<float>(s1);
    p.c_lin = static_cast<float>(q2 + md);
    p.a1_main = static_cast<float>(safety * 2.0 * (gamma_main + 6.0 * kU) * qs);
    p.a1_fp32 = static_cast<float>(safety * 2.0 * (gamma_fp32 + 6.0 * kU) * qs);
    p.a2 = static_cast<float>(safety * (4.02 * kU * qs + 10.11 * kU * md + 4.0 * kU * (q2 + md)) + 1e-6 * md);
    p.a3 = static_cast<float>(safety * (md / 16.0 + 40.0) * kU);
    p.a4 = static_cast<float>(safety * 8.0 * md * md * kE64);
    p.a5 = static_cast<float>(safety * md * kU * kU);
    p.a6 = static_cast<float>(safety * 8.0 * kU * std::fabs(s1));
    p.m = m;
}

// FP32 chain: one FMA per sample and accumulator; split BF16: three products per
// sample plus the tensor-core accumulation (truncating adds, 2^-22 per MMA step).
double gamma_fp32(int m) { return 1.01 * static_cast<double>((m + 63) & ~63) * kU; }
double gamma_bf16(int m) { return 1.2e-5 + (3.0 * ((m + 63) & ~63) / 16.0 + 16.0) * 2.384185791015625e-07; }

// One group of same-length requests of a batch, prepared on the host and resident on
// the device (templates, block orders, epilogue constants).
struct GroupPlan
{
    int m = 0, T = 0, T_pad = 0, m_pad = 0, nblk = 0, nk = 0;
    bool umma_constants = false; // a1_main of the device constants is the tensor-core one
    std::vector<float> a1_umma;  // a1 of the tensor-core kernel per slot
    std::vector<int> index; // request index of each slot
    std::vector<int> mode, k, merge;
    std::vector<float> thr; // threshold distance per slot
    std::vector<TemplParam> htp;
    DevBuf q, order, tp, slots, q_hi, q_lo;
    int t_rows = 0;
    // templates of several lengths (sorted by length, longest first) in 128-row tiles of
    // k_scan_umma or, when col_tile > 0, in column tiles of col_tile rows of k_scan_wm
    bool mixed = false;
    int col_tile = 0;
    bool fft = false; // FFT branch (tm_fft.cu) instead of a contraction kernel
    int k_stride = 0;            // row stride of the template arrays
    uint32_t w_max = 0;          // windows of the shortest template
    std::vector<tmb::TileInfo> tiles; // per tile: K blocks (row tiles: and distinct lengths)
    DevBuf d_tiles;
    void release()
    {
        d_tiles.release();
        q_hi.release();
        q_lo.release();
        q.release();
        order.release();
        tp.release();
        slots.release();
    }
};

} // namespace

struct tm_batch
{
    int count = 0;
    std::vector<GroupPlan> groups;
    uint64_t h2d_bytes = 0;
    ~tm_batch()
    {
        for (GroupPlan &g : groups)
            g.release();
    }
};

namespace {

// Host preparation of one group (bit-identical template z-normalisation and block
// order, epilogue constants) and its upload.
void prepare_group(tm_ctx *ctx, Lane &L, int m, const std::vector<int> &idx, const tm_request *reqs, GroupPlan &g,
                   uint64_t &h2d, int col_tile = 0)
{
    g.m = m;
    g.mixed = false; // a reused plan may have held another kind of group
    g.fft = false;
    g.col_tile = col_tile; // tensor cores: window-major column tiles (k_scan_wm) when > 0
    g.T = static_cast<int>(idx.size());
    g.T_pad = (g.T + 63) & ~63;
    g.m_pad = (m + 63) & ~63;
    g.nblk = std::max(1, m / tm_host::kZnormBlock);
    g.umma_constants = false;
    g.index = idx;
    const int T = g.T, T_pad = g.T_pad, m_pad = g.m_pad, nblk = g.nblk;
    L.h_q.reserve(sizeof(float) * static_cast<size_t>(T_pad) * m_pad);
    L.h_order.reserve(sizeof(int) * static_cast<size_t>(T) * nblk);
    L.h_slots.reserve(sizeof(int) * T);
    float *hq = L.h_q.as<float>();
    int *ho = L.h_order.as<int>();
    int *hslots = L.h_slots.as<int>();
    std::memset(hq, 0, sizeof(float) * static_cast<size_t>(T_pad) * m_pad);
    std::memset(ho, 0, sizeof(int) * static_cast<size_t>(T) * nblk);
    g.htp.assign(T_pad, TemplParam{});
    g.mode.assign(T, 0);
    g.k.assign(T, 0);
    g.merge.assign(T, 0);
    g.thr.assign(T, 0.0f);
    g.a1_umma.assign(T, 0.0f);
    g.nk = 0;
    for (int t = 0; t < T; t++)
    {
        const tm_request *r = &reqs[idx[t]];
        float *q = hq + static_cast<size_t>(t) * m_pad;
        std::memcpy(q, r->templ, sizeof(float) * m);
        if (!(r->flags & TM_FLAG_ZNORMALIZED))
            tm_host::znormalize(q, m);
        tm_host::block_order(q, m, ho + static_cast<size_t>(t) * nblk);
        double q2 = 0.0, s1 = 0.0;
        for (int i = 0; i < m; i++)
        {
            q2 += static_cast<double>(q[i]) * q[i];
            s1 += q[i];
        }
        TemplParam &p = g.htp[t];
        fill_param(p, m, q2, s1, gamma_bf16(m), gamma_fp32(m));
        g.a1_umma[t] = p.a1_main;
        p.a1_main = p.a1_fp32;
        p.mode = g.mode[t] = r->mode;
        p.k = g.k[t] = r->k;
        p.merge = g.merge[t] = r->merge_offset;
        p.q_offset = static_cast<int64_t>(t) * m_pad;
        p.order_offset = static_cast<int64_t>(t) * nblk;
        if (r->mode == TM_MODE_KNN)
            hslots[g.nk++] = t;
        else
            p.thr_ed = g.thr[t] = tm_host::cc_to_ed(r->correlation, m);
    }
    for (int t = T; t < T_pad; t++)
    {
        g.htp[t].mode = TM_MODE_THRESHOLD;
        g.htp[t].thr_ed = -FLT_MAX;
        g.htp[t].m = m;
    }
    cudaStream_t s = L.stream;
    g.q.reserve(sizeof(float) * static_cast<size_t>(T_pad) * m_pad);
    g.order.reserve(sizeof(int) * static_cast<size_t>(T) * nblk);
    g.tp.reserve(sizeof(TemplParam) * T_pad);
    g.slots.reserve(sizeof(int) * std::max(g.nk, 1));
    TM_CUDA(cudaMemcpyAsync(g.q.p, hq, sizeof(float) * static_cast<size_t>(T_pad) * m_pad, cudaMemcpyHostToDevice, s));
    TM_CUDA(cudaMemcpyAsync(g.order.p, ho, sizeof(int) * static_cast<size_t>(T) * nblk, cudaMemcpyHostToDevice, s));
    TM_CUDA(cudaMemcpyAsync(g.tp.p, g.htp.data(), sizeof(TemplParam) * T_pad, cudaMemcpyHostToDevice, s));
    if (g.nk > 0)
        TM_CUDA(cudaMemcpyAsync(g.slots.p, hslots, sizeof(int) * g.nk, cudaMemcpyHostToDevice, s));
    if (ctx->kernel != TM_KERNEL_FP32)
    {
        // BF16 halves for the tensor-core kernel: q = hi + lo (round to nearest even)
        g.t_rows = (T + 127) & ~127;
        const size_t elems = static_cast<size_t>(g.t_rows) * m_pad;
        L.h_split.reserve(2 * sizeof(uint16_t) * elems);
        uint16_t *hh = L.h_split.as<uint16_t>(), *hl = hh + elems;
        std::memset(hh, 0, 2 * sizeof(uint16_t) * elems);
        for (int t = 0; t < T; t++)
            for (int i = 0; i < m; i++)
            {
                const size_t at = static_cast<size_t>(t) * m_pad + i;
                const float v = hq[at];
                hh[at] = bf16_bits(v);
                hl[at] = bf16_bits(v - bf16_value(hh[at]));
            }
        g.q_hi.reserve(sizeof(uint16_t) * elems);
        g.q_lo.reserve(sizeof(uint16_t) * elems);
        TM_CUDA(cudaMemcpyAsync(g.q_hi.p, hh, sizeof(uint16_t) * elems, cudaMemcpyHostToDevice, s));
        TM_CUDA(cudaMemcpyAsync(g.q_lo.p, hl, sizeof(uint16_t) * elems, cudaMemcpyHostToDevice, s));
        h2d += 2 * sizeof(uint16_t) * static_cast<uint64_t>(T) * m;
    }
    // the staging buffers are reused by the next group: finish the copies first
    TM_CUDA(cudaStreamSynchronize(s));
    h2d += sizeof(float) * static_cast<uint64_t>(T) * m + sizeof(int) * static_cast<uint64_t>(T) * nblk +
           sizeof(TemplParam) * T_pad;
}

// Resident FP64 prefix sums and constant-run lengths of the waveform (built once).
void ensure_prefix(tm_ctx *ctx, Lane &L)
{
    if (ctx->prefix_ready)
        return;
    cudaStream_t s = L.stream;
    const uint64_t n = ctx->n;
    const uint32_t chunks = tmb::prefix_chunks(n);
    const uint64_t blocks = (n + tmb::kPrefixBlock - 1) / tmb::kPrefixBlock;
    // zero tail: the contraction kernels read window-end sums in fixed-size chunks that may
    // run past n (values there belong to no window and are never used)
    ctx->prefix.reserve(sizeof(double2) * (n + 1 + tmb::kStagePad));
    TM_CUDA(cudaMemsetAsync(ctx->prefix.p, 0, sizeof(double2) * (n + 1 + tmb::kStagePad), s));
    // one entry past the last block: a window ending at n = blocks x kPrefixBlock reads it
    ctx->ptot.reserve(sizeof(double2) * (blocks + 1));
    ctx->pcen.reserve(sizeof(double) * (blocks + 1));
    TM_CUDA(cudaMemsetAsync(ctx->ptot.p, 0, sizeof(double2) * (blocks + 1), s));
    ctx->run.reserve(sizeof(uint16_t) * n);
    DevBuf totals, run_tmp;
    totals.reserve(sizeof(double2) * chunks);
    run_tmp.reserve(sizeof(uint16_t) * n);
    // centres: the mean of each block, from uncentred chunk sums
    TM_CUDA(tmb::launch_prefix_totals(ctx->clean.as<float>(), n, nullptr, totals.as<double2>(), s));
    std::vector<double2> ct(chunks);
    TM_CUDA(cudaMemcpyAsync(ct.data(), totals.p, sizeof(double2) * chunks, cudaMemcpyDeviceToHost, s));
    TM_CUDA(cudaStreamSynchronize(s));
    const uint64_t per_block = tmb::kPrefixBlock / 8192;
    std::vector<double> centres(blocks + 1, 0.0);
    for (uint64_t b = 0; b < blocks; b++)
    {
        double sum = 0.0;
        for (uint64_t c = b * per_block; c < std::min<uint64_t>(chunks, (b + 1) * per_block); c++)
            sum += ct[c].x;
        const uint64_t count = std::min<uint64_t>(tmb::kPrefixBlock, n - b * tmb::kPrefixBlock);
        centres[b] = sum / static_cast<double>(count);
    }
    centres[blocks] = blocks > 0 ? centres[blocks - 1] : 0.0;
    TM_CUDA(cudaMemcpyAsync(ctx->pcen.p, centres.data(), sizeof(double) * (blocks + 1), cudaMemcpyHostToDevice, s));
    TM_CUDA(tmb::launch_prefix_sums(ctx->clean.as<float>(), n, ctx->pcen.as<double>(), totals.as<double2>(),
                                    ctx->ptot.as<double2>(), ctx->prefix.as<double2>(), s));
    TM_CUDA(tmb::launch_runs(ctx->clean.as<float>(), n, ctx->run.as<uint16_t>(), run_tmp.as<uint16_t>(), s));
    TM_CUDA(cudaStreamSynchronize(s));
    count_launch(L, 4 + 13);
    totals.release();
    run_tmp.release();
    ctx->prefix_ready = true;
}

// Host preparation of a mixed-length group: templates sorted by length (longest first).
// Row tiles (col_tile 0, k_scan_umma): 128 rows, a tile closing early when a new length
// would be its 65th distinct one. Column tiles (k_scan_wm): col_tile rows, any lengths.
// Padding rows are inert; a tile's K extent is its longest template (shorter rows are
// zero-padded, which leaves their dot products unchanged). Rows are the template slots of
// the group: g.index[row] is the request (-1 for padding rows).
void prepare_group_mixed(tm_ctx *ctx, Lane &L, const std::vector<int> &idx_in, const tm_request *reqs, GroupPlan &g,
                         uint64_t &h2d, int col_tile = 0)
{
    std::vector<int> idx = idx_in;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return reqs[a].m > reqs[b].m; });
    const size_t tile_rows = col_tile > 0 ? static_cast<size_t>(col_tile) : 128;
    // rows: request per row (-1 = padding)
    std::vector<int> rows;
    std::vector<tmb::TileInfo> tiles;
    std::vector<int> didx_of_row;
    for (size_t i = 0; i < idx.size();)
    {
        tmb::TileInfo ti{};
        const size_t start = rows.size();
        const int longest = reqs[idx[i]].m;
        while (i < idx.size() && rows.size() - start < tile_rows)
        {
            const int m = reqs[idx[i]].m;
            int d = 0;
            if (col_tile == 0)
            {
                while (d < ti.D && ti.len[d] != m)
                    d++;
                if (d == ti.D)
                {
                    if (ti.D == tmb::kTileLens)
                        break;
                    ti.len[ti.D++] = m;
                }
            }
            rows.push_back(idx[i]);
            didx_of_row.push_back(d);
            i++;
        }
        ti.len[0] = longest;
        ti.kb = (longest + 63) / 64;
        while (rows.size() - start < tile_rows)
        {
            rows.push_back(-1);
            didx_of_row.push_back(0);
        }
        tiles.push_back(ti);
    }
    const int R = static_cast<int>(rows.size()); // multiple of the tile rows
    const int m_max = reqs[idx[0]].m;
    g.mixed = true;
    g.col_tile = col_tile;
    g.fft = false;
    g.m = m_max;
    g.T = R;
    g.T_pad = R;
    g.t_rows = R;
    g.k_stride = (m_max + 63) & ~63;
    g.m_pad = g.k_stride;
    g.nblk = std::max(1, g.k_stride / tm_host::kZnormBlock);
    g.umma_constants = true;
    g.index = rows;
    const int stride = g.k_stride, nblk = g.nblk;
    const size_t elems = static_cast<size_t>(R) * stride;
    L.h_q.reserve(sizeof(float) * elems);
    L.h_order.reserve(sizeof(int) * static_cast<size_t>(R) * nblk);
    L.h_slots.reserve(sizeof(int) * R);
    L.h_split.reserve(2 * sizeof(uint16_t) * elems);
    float *hq = L.h_q.as<float>();
    int *ho = L.h_order.as<int>();
    int *hslots = L.h_slots.as<int>();
    uint16_t *hh = L.h_split.as<uint16_t>(), *hl = hh + elems;
    std::memset(hq, 0, sizeof(float) * elems);
    std::memset(ho, 0, sizeof(int) * static_cast<size_t>(R) * nblk);
    std::memset(hh, 0, 2 * sizeof(uint16_t) * elems);
    g.htp.assign(R, TemplParam{});
    g.mode.assign(R, TM_MODE_THRESHOLD);
    g.k.assign(R, 0);
    g.merge.assign(R, 0);
    g.thr.assign(R, -FLT_MAX);
    g.a1_umma.assign(R, 0.0f);
    g.nk = 0;
    g.w_max = 0;
    const uint64_t w0 = ctx->range_first;
    auto wcount_of = [&](int m) {
        const uint64_t total = ctx->n - static_cast<uint64_t>(m) + 1;
        return static_cast<uint32_t>(w0 >= total ? 0 : std::min<uint64_t>(ctx->range_count, total - w0));
    };
    uint64_t samples = 0;
    for (int t = 0; t < R; t++)
    {
        TemplParam &p = g.htp[t];
        const tmb::TileInfo &ti = tiles[static_cast<size_t>(t) / tile_rows];
        p.didx = didx_of_row[t];
        if (rows[t] < 0)
        {
            p.mode = TM_MODE_THRESHOLD;
            p.thr_ed = -FLT_MAX;
            p.m = ti.len[0];
            p.inv_m = 1.0 / p.m;
            p.wcount = 0;
            continue;
        }
        const tm_request *r = &reqs[rows[t]];
        const int m = r->m;
        samples += static_cast<uint64_t>(m);
        float *q = hq + static_cast<size_t>(t) * stride;
        std::memcpy(q, r->templ, sizeof(float) * m);
        if (!(r->flags & TM_FLAG_ZNORMALIZED))
            tm_host::znormalize(q, m);
        tm_host::block_order(q, m, ho + static_cast<size_t>(t) * nblk);
        double q2 = 0.0, s1 = 0.0;
        for (int i = 0; i < m; i++)
        {
            q2 += static_cast<double>(q[i]) * q[i];
            s1 += q[i];
            const size_t at = static_cast<size_t>(t) * stride + i;
            hh[at] = bf16_bits(q[i]);
            hl[at] = bf16_bits(q[i] - bf16_value(hh[at]));
        }
        fill_param(p, m, q2, s1, gamma_bf16(m), gamma_fp32(m));
        g.a1_umma[t] = p.a1_main;
        p.inv_m = 1.0 / static_cast<double>(m);
        p.qs = static_cast<float>(std::sqrt(q2 * m));
        p.wcount = wcount_of(m);
        g.w_max = std::max(g.w_max, p.wcount);
        p.mode = g.mode[t] = r->mode;
        p.k = g.k[t] = r->k;
        p.merge = g.merge[t] = r->merge_offset;
        p.q_offset = static_cast<int64_t>(t) * stride;
        p.order_offset = static_cast<int64_t>(t) * nblk;
        if (r->mode == TM_MODE_KNN)
            hslots[g.nk++] = t;
        else
            p.thr_ed = g.thr[t] = tm_host::cc_to_ed(r->correlation, m);
    }
    for (tmb::TileInfo &ti : tiles)
        for (int d = 0; d < ti.D; d++)
        {
            ti.wc[d] = wcount_of(ti.len[d]);
            ti.inv_m[d] = 1.0 / static_cast<double>(ti.len[d]);
        }
    g.tiles = tiles;
    cudaStream_t s = L.stream;
    g.q.reserve(sizeof(float) * elems);
    g.order.reserve(sizeof(int) * static_cast<size_t>(R) * nblk);
    g.tp.reserve(sizeof(TemplParam) * R);
    g.slots.reserve(sizeof(int) * std::max(g.nk, 1));
    g.q_hi.reserve(sizeof(uint16_t) * elems);
    g.q_lo.reserve(sizeof(uint16_t) * elems);
    g.d_tiles.reserve(sizeof(tmb::TileInfo) * tiles.size());
    TM_CUDA(cudaMemcpyAsync(g.q.p, hq, sizeof(float) * elems, cudaMemcpyHostToDevice, s));
    TM_CUDA(cudaMemcpyAsync(g.order.p, ho, sizeof(int) * static_cast<size_t>(R) * nblk, cudaMemcpyHostToDevice, s));
    TM_CUDA(cudaMemcpyAsync(g.tp.p, g.htp.data(), sizeof(TemplParam) * R, cudaMemcpyHostToDevice, s));
    if (g.nk > 0)
        TM_CUDA(cudaMemcpyAsync(g.slots.p, hslots, sizeof(int) * g.nk, cudaMemcpyHostToDevice, s));
    TM_CUDA(cudaMemcpyAsync(g.q_hi.p, hh, sizeof(uint16_t) * elems, cudaMemcpyHostToDevice, s));
    TM_CUDA(cudaMemcpyAsync(g.q_lo.p, hl, sizeof(uint16_t) * elems, cudaMemcpyHostToDevice, s));
    TM_CUDA(cudaMemcpyAsync(g.d_tiles.p, g.tiles.data(), sizeof(tmb::TileInfo) * tiles.size(), cudaMemcpyHostToDevice,
                            s));
    TM_CUDA(cudaStreamSynchronize(s));
    h2d += samples * (sizeof(float) + 2 * sizeof(uint16_t)) + sizeof(int) * static_cast<uint64_t>(R) * nblk +
           sizeof(TemplParam) * R + sizeof(tmb::TileInfo) * tiles.size();
}

// A pinned block of at least `need` bytes that no result holds, from the pool or new.
std::shared_ptr<PinnedBlock> acquire_block(Lane &L, size_t need)
{
    auto &pool = L.pool;
    for (auto &b : pool)
        if (b.use_count() == 1 && b->bytes >= need)
            return b;
    pool.erase(std::remove_if(pool.begin(), pool.end(),
                              [](const std::shared_ptr<PinnedBlock> &b) { return b.use_count() == 1; }),
               pool.end());
    pool.push_back(std::make_shared<PinnedBlock>(std::max<size_t>(need + need / 4, 1u << 20)));
    return pool.back();
}

// Largest k whose selection runs on the device (k_select_knn keeps k windows per warp in
// shared memory); groups with a larger k select on the host.
constexpr int kMaxDeviceK = 1024;

// What the device left for a group's answers (host pointers into the pinned block,
// device pointers for the runs that stay on the device).
struct AnswerView
{
    uint32_t *win = nullptr; // threshold runs: windows relative to w0, then ED^2
    float *dist = nullptr;
    const uint32_t *start = nullptr, *end = nullptr, *tkey = nullptr;
    bool device_knn = false; // kNN selections made by k_select_knn:
    int kcap = 0;            //   slot s: knn_n[s] answers at s * kcap
    const uint32_t *knn_n = nullptr, *knn_win = nullptr;
    const float *knn_dist = nullptr;
    const uint32_t *d_win = nullptr; // the sorted runs on the device
    const float *d_dist = nullptr;
};

// Canonical answers of each template of a group.
// Threshold: the template's run (position order, no repeats), thinned in place by the
// merge offset. kNN: the device's exclusion selection over the finite distances. When
// that leaves fewer than k answers and the bound was unbounded (too few separated
// windows for the reference's queue to fill), or k is too large for the device, the
// template's run (in (distance, position) order) is fetched and selected here: the
// windows of distance FLT_MAX (constant windows, which the contraction skips, plus any
// re-scored to FLT_MAX) follow the finite ones in position order, as in the reference.
template <class Degenerate>
void finish_answers(Lane &L, const GroupPlan &g, const AnswerView &v, uint64_t w0, tm_result &res,
                    Degenerate degenerate_windows)
{
    int slot = -1;
    for (int t = 0; t < g.T; t++)
    {
        const bool knn = g.mode[t] == TM_MODE_KNN;
        slot += knn ? 1 : 0;
        if (g.index[t] < 0)
            continue; // padding row of a mixed-length tile
        Answer &out = res.answers[g.index[t]];
        const uint32_t a = v.start[t], b = v.end[t];
        if (!knn)
        {
            uint32_t count = b - a;
            if (g.merge[t] > 0) // SkipSequential.cpp:358-370: skip pos < last kept + merge + 1
            {
                const uint64_t gap = static_cast<uint64_t>(g.merge[t]) + 1;
                uint32_t w = a;
                for (uint32_t i = a; i < b; i++)
                {
                    if (w > a && static_cast<uint64_t>(v.win[i]) < static_cast<uint64_t>(v.win[w - 1]) + gap)
                        continue;
                    v.win[w] = v.win[i];
                    v.dist[w] = v.dist[i];
                    w++;
                }
                count = w - a;
            }
            out.hits.clear();
            out.run = true;
            out.win = v.win + a;
            out.dist = v.dist + a;
            out.w0 = w0;
            out.count = count;
            continue;
        }
        std::vector<Hit> kept;
        const bool unbounded = v.tkey[t] == tmb::kEmptyKey;
        if (v.device_knn && (static_cast<int>(v.knn_n[slot]) >= g.k[t] || !unbounded))
        {
            const size_t at = static_cast<size_t>(slot) * v.kcap;
            for (uint32_t i = 0; i < v.knn_n[slot]; i++)
                kept.push_back(Hit{w0 + v.knn_win[at + i], v.knn_dist[at + i]});
        }
        else
        {
            std::vector<uint32_t> rw(b - a);
            std::vector<float> rd(b - a);
            if (b > a)
            {
                TM_CUDA(cudaMemcpyAsync(rw.data(), v.d_win + a, sizeof(uint32_t) * (b - a), cudaMemcpyDeviceToHost,
                                        L.stream));
                TM_CUDA(cudaMemcpyAsync(rd.data(), v.d_dist + a, sizeof(float) * (b - a), cudaMemcpyDeviceToHost,
                                        L.stream));
                TM_CUDA(cudaStreamSynchronize(L.stream));
                L.d2h_bytes += 8ull * (b - a);
            }
            std::vector<Hit> finite, infinite;
            for (uint32_t i = 0; i < b - a; i++)
                (rd[i] < FLT_MAX ? finite : infinite).push_back(Hit{w0 + rw[i], rd[i]});
            tm_host::select_knn(finite, g.k[t], g.merge[t], kept);
            if (static_cast<int>(kept.size()) < g.k[t] && unbounded)
            {
                degenerate_windows(t, infinite);
                std::sort(infinite.begin(), infinite.end(), [](const Hit &x, const Hit &y) { return x.pos < y.pos; });
                infinite.erase(std::unique(infinite.begin(), infinite.end(),
                                           [](const Hit &x, const Hit &y) { return x.pos == y.pos; }),
                               infinite.end());
                tm_host::extend_knn(infinite, g.k[t], g.merge[t], kept);
            }
        }
        while (static_cast<int>(kept.size()) < g.k[t])
            kept.push_back(Hit{0, FLT_MAX});
        out.set_hits(std::move(kept));
    }
}

void add_span(Lane &L, int phase, cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.0f;
    TM_CUDA(cudaEventElapsedTime(&ms, a, b));
    L.phase_ms[phase] += ms;
}

// Exact re-scoring of a group's ncand candidates, answer order and kNN selection on the
// device, one copy to a pinned block that the result keeps, canonical answers.
template <class Degenerate>
void rescore_and_answer(tm_ctx *ctx, Lane &L, const GroupPlan &g, uint32_t ncand, uint64_t w0, tm_result &res,
                        Degenerate degenerate_windows)
{
    cudaStream_t s = L.stream;
    const int T = g.T, nk = g.nk;
    int kcap = 1;
    for (int t = 0; t < T; t++)
        if (g.mode[t] == TM_MODE_KNN)
            kcap = std::max(kcap, g.k[t]);
    const bool device_knn = nk > 0 && kcap <= kMaxDeviceK;
    const size_t cn = std::max<uint32_t>(ncand, 1);
    L.dist.reserve(sizeof(float) * cn);
    L.akeys.reserve(2 * sizeof(unsigned long long) * cn);
    L.avals.reserve(2 * sizeof(float) * cn);
    if (nk > 0)
        L.avals64.reserve(2 * sizeof(unsigned long long) * cn);
    L.segs.reserve(sizeof(uint32_t) * (2 * static_cast<size_t>(std::max(T, 1)) +
                                          (device_knn ? static_cast<size_t>(nk) * (1 + 2 * kcap) : 0)));
    uint32_t *hc = L.h_counters.as<uint32_t>();
    uint32_t *d_kept = L.counters.as<uint32_t>() + 3;
    if (L.profile)
        TM_CUDA(cudaEventRecord(L.ev2, s));
    TM_CUDA(tmb::launch_rescore(L.cand.as<Candidate>(), ncand, g.tp.as<TemplParam>(), g.q.as<float>(),
                                g.order.as<int>(), ctx->raw.as<float>(), w0, L.dist.as<float>(), s));
    if (ncand > 0)
        count_launch(L);
    if (L.profile)
        TM_CUDA(cudaEventRecord(L.ev3, s));
    unsigned long long *keys[2] = {L.akeys.as<unsigned long long>(), L.akeys.as<unsigned long long>() + cn};
    float *vals32[2] = {L.avals.as<float>(), L.avals.as<float>() + cn};
    unsigned long long *vals64[2] = {L.avals64.as<unsigned long long>(),
                                     L.avals64.as<unsigned long long>() + (nk > 0 ? cn : 0)};
    TM_CUDA(cudaMemsetAsync(d_kept, 0, 2 * sizeof(uint32_t), s));
    TM_CUDA(tmb::launch_answer_keys(L.cand.as<Candidate>(), L.dist.as<float>(), ncand, g.tp.as<TemplParam>(),
                                    keys[0], vals32[0], d_kept, s));
    TM_CUDA(cudaMemcpyAsync(hc + 3, d_kept, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    TM_CUDA(cudaStreamSynchronize(s));
    if (ncand > 0)
        count_launch(L);
    const uint32_t kept = hc[3], knn_kept = hc[4], thr_kept = kept - knn_kept;
    const size_t scratch = tmb::answer_sort_scratch(kept, T);
    L.sort_tmp.reserve(scratch);
    uint32_t *d_start = L.segs.as<uint32_t>(), *d_end = d_start + T;
    uint32_t *d_knn_n = d_end + T, *d_knn_win = d_knn_n + nk;
    float *d_knn_dist = reinterpret_cast<float *>(d_knn_win + static_cast<size_t>(nk) * kcap);
    uint32_t *d_win = reinterpret_cast<uint32_t *>(L.cand.p); // the candidates are consumed: reuse
    float *d_dist = L.dist.as<float>();                       // likewise the re-scored distances
    TM_CUDA(cudaMemsetAsync(d_start, 0, 2 * sizeof(uint32_t) * T, s));
    TM_CUDA(tmb::launch_answer_order(keys, vals32, vals64, kept, knn_kept, g.tp.as<TemplParam>(), T, L.sort_tmp.p,
                                     scratch, d_start, d_end, d_win, d_dist, s));
    if (kept > 0)
        count_launch(L, knn_kept > 0 ? 4 : 2); // each radix sort counted as one launch
    if (device_knn)
    {
        TM_CUDA(tmb::launch_select_knn(g.slots.as<int>(), nk, g.tp.as<TemplParam>(), d_start, d_end, d_win, d_dist,
                                       kcap, d_knn_n, d_knn_win, d_knn_dist, s));
        count_launch(L);
    }
    if (L.profile)
        TM_CUDA(cudaEventRecord(L.ev4, s));

    // block layout: win[thr_kept] | dist[thr_kept] | start[T] | end[T] | tkey[T] |
    //               knn_n[nk] | knn_win[nk * kcap] | knn_dist[nk * kcap]
    const size_t knn_words = device_knn ? static_cast<size_t>(nk) * (1 + 2 * kcap) : 0;
    std::shared_ptr<PinnedBlock> block = acquire_block(
        L, sizeof(uint32_t) * (2 * static_cast<size_t>(thr_kept) + 3 * static_cast<size_t>(T) + knn_words) + 64);
    AnswerView v;
    v.win = static_cast<uint32_t *>(block->p);
    v.dist = reinterpret_cast<float *>(v.win + thr_kept);
    uint32_t *h_start = reinterpret_cast<uint32_t *>(v.dist + thr_kept);
    uint32_t *h_tkey = h_start + 2 * static_cast<size_t>(T);
    uint32_t *h_knn = h_tkey + T;
    if (thr_kept > 0)
    {
        TM_CUDA(cudaMemcpyAsync(v.win, d_win, sizeof(uint32_t) * thr_kept, cudaMemcpyDeviceToHost, s));
        TM_CUDA(cudaMemcpyAsync(v.dist, d_dist, sizeof(float) * thr_kept, cudaMemcpyDeviceToHost, s));
    }
    TM_CUDA(cudaMemcpyAsync(h_start, d_start, 2 * sizeof(uint32_t) * T, cudaMemcpyDeviceToHost, s));
    if (nk > 0)
        TM_CUDA(cudaMemcpyAsync(h_tkey, L.tkey.p, sizeof(uint32_t) * T, cudaMemcpyDeviceToHost, s));
    else
        std::fill(h_tkey, h_tkey + T, 0u);
    if (device_knn)
        TM_CUDA(cudaMemcpyAsync(h_knn, d_knn_n, sizeof(uint32_t) * knn_words, cudaMemcpyDeviceToHost, s));
    if (L.profile)
        TM_CUDA(cudaEventRecord(L.ev1, s));
    TM_CUDA(cudaStreamSynchronize(s));
    L.last_candidates += ncand;
    L.d2h_bytes += sizeof(uint32_t) * (2 * static_cast<uint64_t>(thr_kept) + 2 * static_cast<uint64_t>(T) +
                                          (nk > 0 ? T : 0) + knn_words) +
                      16;
    const auto t0 = std::chrono::steady_clock::now();
    if (L.profile)
    {
        add_span(L, 2, L.ev2, L.ev3);
        add_span(L, 3, L.ev3, L.ev4);
        add_span(L, 4, L.ev4, L.ev1);
    }
    v.start = h_start;
    v.end = h_start + T;
    v.tkey = h_tkey;
    v.device_knn = device_knn;
    v.kcap = kcap;
    v.knn_n = h_knn;
    v.knn_win = h_knn + nk;
    v.knn_dist = reinterpret_cast<const float *>(h_knn + nk + static_cast<size_t>(nk) * kcap);
    v.d_win = d_win;
    v.d_dist = d_dist;
    res.blocks.push_back(block);
    finish_answers(L, g, v, w0, res, degenerate_windows);
    if (L.profile)
        L.phase_ms[5] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Device pipeline and selection for one prepared group; writes answers[index].
void execute_group(tm_ctx *ctx, Lane &L, GroupPlan &g, tm_result &res)
{
    const int m = g.m;
    LengthStats &ls = ensure_length(ctx, L, m);
    const int T = g.T, T_pad = g.T_pad, m_pad = g.m_pad, nk = g.nk;
    const uint64_t w0 = ls.w0, W = ls.W;
    if (W == 0)
    {
        for (int t = 0; t < T; t++)
            res.answers[g.index[t]].set_hits(g.mode[t] == TM_MODE_KNN
                                                 ? std::vector<Hit>(static_cast<size_t>(g.k[t]), Hit{0, FLT_MAX})
                                                 : std::vector<Hit>());
        return;
    }
    if (W >= (1ull << 32))
        throw Failure{TM_ERR_ARGUMENT, "more than 2^32 - 1 windows in one range; split the range"};
    cudaStream_t s = L.stream;
    const bool use_umma = ctx->kernel != TM_KERNEL_FP32 && g.t_rows > 0 && tmb::umma_supported(m, T, W);
    if (ctx->kernel == TM_KERNEL_SPLIT_BF16 && !use_umma)
        throw Failure{TM_ERR_STATE, "split-BF16 kernel not available for this request group"};
    if (use_umma != g.umma_constants) // error-bound constants of the kernel that will run
    {
        for (int t = 0; t < T; t++)
            g.htp[t].a1_main = use_umma ? g.a1_umma[t] : g.htp[t].a1_fp32;
        TM_CUDA(cudaMemcpyAsync(g.tp.p, g.htp.data(), sizeof(TemplParam) * T_pad, cudaMemcpyHostToDevice, s));
        g.umma_constants = use_umma;
    }
    L.tkey.reserve(sizeof(uint32_t) * T);

    const uint32_t nb = static_cast<uint32_t>((W + tmb::kBucket - 1) / tmb::kBucket);
    if (nk > 0)
    {
        L.bmin_u.reserve(sizeof(uint32_t) * static_cast<size_t>(T) * nb);
        L.bmin_l.reserve(sizeof(uint32_t) * static_cast<size_t>(T) * nb);
    }
    L.counters.reserve(8 * sizeof(uint32_t));
    L.h_counters.reserve(8 * sizeof(uint32_t));
    uint32_t *hc = L.h_counters.as<uint32_t>();

    uint32_t ncand = 0;
    for (int attempt = 0; attempt < 3; attempt++)
    {
        L.cand.reserve(sizeof(Candidate) * static_cast<size_t>(L.cand_cap));
        if (nk > 0)
        {
            TM_CUDA(cudaMemsetAsync(L.bmin_u.p, 0xff, sizeof(uint32_t) * static_cast<size_t>(T) * nb, s));
            TM_CUDA(cudaMemsetAsync(L.bmin_l.p, 0xff, sizeof(uint32_t) * static_cast<size_t>(T) * nb, s));
        }
        TM_CUDA(cudaMemsetAsync(L.counters.p, 0, 4 * sizeof(uint32_t), s));
        uint32_t *d_cand_count = L.counters.as<uint32_t>();
        uint32_t *d_list_count = d_cand_count + 1;

        tmb::ScanArgs a{};
        a.x = ctx->clean.as<float>();
        a.q = g.q.as<float>();
        a.tp = g.tp.as<TemplParam>();
        a.mean = ls.mean.as<float>();
        a.inv = ls.inv.as<float>();
        a.w0 = w0;
        a.W = static_cast<uint32_t>(W);
        a.m_pad = m_pad;
        a.T = T;
        a.bmin_u = L.bmin_u.as<uint32_t>();
        a.bmin_l = L.bmin_l.as<uint32_t>();
        a.nb = nb;
        a.cand = L.cand.as<Candidate>();
        a.cand_count = d_cand_count;
        a.cand_cap = L.cand_cap;
        a.q_hi = g.q_hi.p;
        a.q_lo = g.q_lo.p;
        a.t_rows = g.t_rows;
        a.err = reinterpret_cast<int *>(d_cand_count + 2);

        // 2. contraction with fused epilogue
        if (L.profile)
            TM_CUDA(cudaEventRecord(L.ev0, s));
        a.col_tile = g.col_tile;
        if (use_umma)
            TM_CUDA(g.col_tile > 0 ? tmb::launch_scan_wm(a, s) : tmb::launch_scan_umma(a, s));
        else
            TM_CUDA(tmb::launch_scan_fp32(a, s));
        count_launch(L);
        if (L.profile)
        {
            TM_CUDA(cudaEventRecord(L.ev1, s));
            TM_CUDA(cudaEventSynchronize(L.ev1));
            float ms = 0.0f;
            TM_CUDA(cudaEventElapsedTime(&ms, L.ev0, L.ev1));
            L.kname = use_umma ? (g.col_tile > 0 ? "k_scan_wm" : "k_scan_umma") : "k_scan_fp32";
            L.prof_launches++;
            L.prof_ms += ms;
            L.phase_ms[0] += ms;
            L.prof_flops += 2.0 * m * static_cast<double>(W) * T;
        }

        // 3. kNN bound, bucket list, FP32 re-pass
        if (nk > 0)
        {
            TM_CUDA(tmb::launch_bucket_select(L.bmin_u.as<uint32_t>(), nb, g.tp.as<TemplParam>(),
                                              g.slots.as<int>(), nk, L.tkey.as<uint32_t>(), s));
            for (int la = 0; la < 3; la++)
            {
                L.list.reserve(sizeof(uint2) * static_cast<size_t>(L.list_cap));
                TM_CUDA(cudaMemsetAsync(d_list_count, 0, sizeof(uint32_t), s));
                TM_CUDA(tmb::launch_list_buckets(L.bmin_l.as<uint32_t>(), nb, g.slots.as<int>(), nk,
                                                 L.tkey.as<uint32_t>(), L.list.as<uint2>(), d_list_count,
                                                 L.list_cap, s));
                TM_CUDA(cudaMemcpyAsync(hc + 1, d_list_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
                TM_CUDA(cudaStreamSynchronize(s));
                count_launch(L, 2);
                if (hc[1] <= L.list_cap)
                    break;
                L.list_cap = hc[1] + hc[1] / 2;
            }
            if (hc[1] > L.list_cap)
                throw Failure{TM_ERR_NO_MEMORY, "bucket list overflow"};
            TM_CUDA(tmb::launch_passb(L.list.as<uint2>(), hc[1], ctx->clean.as<float>(), g.q.as<float>(),
                                      g.tp.as<TemplParam>(), ls.mean.as<float>(), ls.inv.as<float>(),
                                      L.tkey.as<uint32_t>(), w0, static_cast<uint32_t>(W),
                                      L.cand.as<Candidate>(), d_cand_count, L.cand_cap, s));
            if (hc[1] > 0)
                count_launch(L);
        }
        if (L.profile)
            TM_CUDA(cudaEventRecord(L.ev2, s));
        TM_CUDA(cudaMemcpyAsync(hc, d_cand_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        TM_CUDA(cudaMemcpyAsync(hc + 2, d_cand_count + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        TM_CUDA(cudaStreamSynchronize(s));
        if (L.profile)
            add_span(L, 1, L.ev1, L.ev2);
        if (hc[2] != 0)
            throw Failure{TM_ERR_TIMEOUT, "contraction kernel gave up waiting (code " + std::to_string(hc[2]) + ")"};
        ncand = hc[0];
        if (ncand <= L.cand_cap)
            break;
        L.cand_cap = ncand + ncand / 2;
        if (attempt == 2)
            throw Failure{TM_ERR_NO_MEMORY, "candidate buffer overflow"};
    }

    std::vector<uint8_t> flags; // fetched only when some kNN bound is unbounded
    rescore_and_answer(ctx, L, g, ncand, w0, res, [&](int, std::vector<Hit> &degenerate) {
        if (flags.empty())
        {
            flags.resize(W);
            TM_CUDA(cudaMemcpy(flags.data(), ls.flags.p, W, cudaMemcpyDeviceToHost));
        }
        for (uint64_t j = 0; j < W; j++)
            if ((flags[j] & tmb::kFlagDegenerate) && !(flags[j] & tmb::kFlagMissingStart))
                degenerate.push_back(Hit{w0 + j, FLT_MAX});
    });
}

#define TM_CUFFT(call)                                                                                            \
    do                                                                                                            \
    {                                                                                                             \
        const cufftResult r_ = (call);                                                                            \
        if (r_ != CUFFT_SUCCESS)                                                                                  \
            throw Failure{r_ == CUFFT_ALLOC_FAILED ? TM_ERR_NO_MEMORY : TM_ERR_CUDA,                             \
                          std::string(#call) + ": cuFFT error " + std::to_string(static_cast<int>(r_))};         \
    } while (0)

// Spectra of the record's overlapping pieces (tm_fft.cu), their shifts and norms: built
// once per context (under a lock: serving workers may ask at once).
void ensure_fft(tm_ctx *ctx, Lane &L)
{
    std::lock_guard<std::mutex> lk(ctx->fft_mu);
    if (ctx->fft_ready)
        return;
    ensure_prefix(ctx, L);
    cudaStream_t s = L.stream;
    const uint32_t P = tmb::fft_pieces(ctx->n);
    const uint32_t B = tmb::kFftBatch;
    const uint64_t Ppad = (static_cast<uint64_t>(P) + B - 1) / B * B; // whole batches; extra pieces stay zero
    ctx->fft_X.reserve(sizeof(double2) * Ppad * tmb::kFftH);
    ctx->fft_shift.reserve(sizeof(double) * Ppad);
    ctx->fft_norm.reserve(sizeof(double) * Ppad);
    TM_CUDA(cudaMemsetAsync(ctx->fft_X.p, 0, sizeof(double2) * Ppad * tmb::kFftH, s));
    TM_CUDA(cudaMemsetAsync(ctx->fft_shift.p, 0, sizeof(double) * Ppad, s));
    TM_CUDA(cudaMemsetAsync(ctx->fft_norm.p, 0, sizeof(double) * Ppad, s));
    DevBuf pieces;
    pieces.reserve(sizeof(double) * static_cast<size_t>(B) * tmb::kFftL);
    cufftHandle plan;
    int len = tmb::kFftL;
    TM_CUFFT(cufftPlanMany(&plan, 1, &len, nullptr, 1, tmb::kFftL, nullptr, 1, tmb::kFftH, CUFFT_D2Z,
                           static_cast<int>(B)));
    std::unique_ptr<cufftHandle, void (*)(cufftHandle *)> hold(&plan, [](cufftHandle *h) { cufftDestroy(*h); });
    TM_CUFFT(cufftSetStream(plan, s));
    for (uint32_t p0 = 0; p0 < P; p0 += B)
    {
        const uint32_t cnt = std::min<uint32_t>(B, P - p0);
        if (cnt < B)
            TM_CUDA(cudaMemsetAsync(pieces.p, 0, sizeof(double) * static_cast<size_t>(B) * tmb::kFftL, s));
        TM_CUDA(tmb::launch_fft_gather(ctx->clean.as<float>(), ctx->n, ctx->pcen.as<double>(), p0, cnt,
                                       pieces.as<double>(), ctx->fft_shift.as<double>(), ctx->fft_norm.as<double>(),
                                       s));
        TM_CUFFT(cufftExecD2Z(plan, pieces.as<cufftDoubleReal>(),
                              reinterpret_cast<cufftDoubleComplex *>(ctx->fft_X.as<double2>() +
                                                                     static_cast<size_t>(p0) * tmb::kFftH)));
        count_launch(L, 2);
    }
    TM_CUDA(cudaStreamSynchronize(s));
    pieces.release();
    ctx->fft_P = P;
    ctx->fft_ready = true;
}

// The lane's FFT plans and buffers.
void ensure_lane_fft(Lane &L)
{
    if (L.fft_plans)
        return;
    int len = tmb::kFftL;
    TM_CUFFT(cufftPlan1d(&L.fft_plan1, tmb::kFftL, CUFFT_D2Z, 1));
    if (cufftPlanMany(&L.fft_planB, 1, &len, nullptr, 1, tmb::kFftH, nullptr, 1, tmb::kFftL, CUFFT_Z2D,
                      static_cast<int>(tmb::kFftBatch)) != CUFFT_SUCCESS)
    {
        cufftDestroy(L.fft_plan1);
        throw Failure{TM_ERR_CUDA, "cufftPlanMany (inverse FFT batch) failed"};
    }
    L.fft_plans = true;
    TM_CUFFT(cufftSetStream(L.fft_plan1, L.stream));
    TM_CUFFT(cufftSetStream(L.fft_planB, L.stream));
    L.fft_y.reserve(sizeof(double) * tmb::kFftL);
    L.fft_Y.reserve(sizeof(double2) * tmb::kFftH);
    L.fft_Z.reserve(sizeof(double2) * static_cast<size_t>(tmb::kFftBatch) * tmb::kFftH);
    L.fft_out.reserve(sizeof(double) * static_cast<size_t>(tmb::kFftBatch) * tmb::kFftL);
}

// FFT branch of a prepared mixed-length group: each template's correlation with every
// piece its windows touch, batch by batch, into the same bucket minima and candidate
// list as the contraction kernels (a: the launch arguments those would get).
void fft_contract(tm_ctx *ctx, Lane &L, const GroupPlan &g, const tmb::ScanArgs &a)
{
    ensure_fft(ctx, L);
    ensure_lane_fft(L);
    cudaStream_t s = L.stream;
    const uint32_t B = tmb::kFftBatch, P = ctx->fft_P;
    for (int t = 0; t < g.T; t++)
    {
        const TemplParam &p = g.htp[t];
        if (g.index[t] < 0 || p.wcount == 0)
            continue;
        TM_CUDA(tmb::launch_fft_template(g.q.as<float>() + p.q_offset, p.m, L.fft_y.as<double>(), s));
        TM_CUFFT(cufftExecD2Z(L.fft_plan1, L.fft_y.as<cufftDoubleReal>(),
                              reinterpret_cast<cufftDoubleComplex *>(L.fft_Y.p)));
        const uint64_t first = a.w0, last = a.w0 + p.wcount - 1;
        const uint32_t pa = static_cast<uint32_t>(first / tmb::kFftS), pb = static_cast<uint32_t>(last / tmb::kFftS);
        for (uint32_t p0 = pa / B * B; p0 <= pb && p0 < P; p0 += B)
        {
            TM_CUDA(tmb::launch_fft_mul(ctx->fft_X.as<double2>() + static_cast<size_t>(p0) * tmb::kFftH,
                                        L.fft_Y.as<double2>(), L.fft_Z.as<double2>(), B, s));
            TM_CUFFT(cufftExecZ2D(L.fft_planB, reinterpret_cast<cufftDoubleComplex *>(L.fft_Z.p),
                                  L.fft_out.as<cufftDoubleReal>()));
            tmb::FftEpiArgs f{};
            f.out = L.fft_out.as<double>();
            f.p0 = p0;
            f.count = std::min<uint32_t>(B, P - p0);
            f.t = static_cast<uint32_t>(t);
            f.tp = g.tp.as<TemplParam>();
            f.w0 = a.w0;
            f.pv = tmb::PrefixView{a.P, a.PT, a.PC};
            f.run = a.run;
            f.raw = a.raw;
            f.shifts = ctx->fft_shift.as<double>();
            f.norms = ctx->fft_norm.as<double>();
            f.bmin_u = a.bmin_u;
            f.bmin_l = a.bmin_l;
            f.nb = a.nb;
            f.cand = a.cand;
            f.cand_count = a.cand_count;
            f.cand_cap = a.cand_cap;
            f.dbg_d = a.dbg_d;
            f.dbg_e = a.dbg_e;
            f.W = a.W;
            TM_CUDA(tmb::launch_fft_epilogue(f, s));
            count_launch(L, 3);
        }
        count_launch(L, 2);
    }
}

// Device pipeline for a mixed-length group (tensor-core kernels or the FFT branch).
void execute_group_mixed(tm_ctx *ctx, Lane &L, GroupPlan &g, tm_result &res)
{
    if (ctx->kernel == TM_KERNEL_FP32 && !g.fft)
        throw Failure{TM_ERR_STATE, "batch of several template lengths was prepared for the tensor-core kernel"};
    ensure_prefix(ctx, L);
    const int T = g.T, nk = g.nk;
    const uint64_t w0 = ctx->range_first, W = g.w_max;
    if (W == 0)
    {
        for (int t = 0; t < T; t++)
            if (g.index[t] >= 0)
                res.answers[g.index[t]].set_hits(g.mode[t] == TM_MODE_KNN
                                                     ? std::vector<Hit>(static_cast<size_t>(g.k[t]), Hit{0, FLT_MAX})
                                                     : std::vector<Hit>());
        return;
    }
    if (W >= (1ull << 32))
        throw Failure{TM_ERR_ARGUMENT, "more than 2^32 - 1 windows in one range; split the range"};
    cudaStream_t s = L.stream;
    L.tkey.reserve(sizeof(uint32_t) * T);
    const uint32_t nb = static_cast<uint32_t>((W + tmb::kBucket - 1) / tmb::kBucket);
    if (nk > 0)
    {
        L.bmin_u.reserve(sizeof(uint32_t) * static_cast<size_t>(T) * nb);
        L.bmin_l.reserve(sizeof(uint32_t) * static_cast<size_t>(T) * nb);
    }
    L.counters.reserve(8 * sizeof(uint32_t));
    L.h_counters.reserve(8 * sizeof(uint32_t));
    uint32_t *hc = L.h_counters.as<uint32_t>();
    double flops = 0.0;
    for (int t = 0; t < T; t++)
        flops += 2.0 * g.htp[t].m * static_cast<double>(g.htp[t].wcount);

    uint32_t ncand = 0;
    for (int attempt = 0; attempt < 3; attempt++)
    {
        L.cand.reserve(sizeof(Candidate) * static_cast<size_t>(L.cand_cap));
        if (nk > 0)
        {
            TM_CUDA(cudaMemsetAsync(L.bmin_u.p, 0xff, sizeof(uint32_t) * static_cast<size_t>(T) * nb, s));
            TM_CUDA(cudaMemsetAsync(L.bmin_l.p, 0xff, sizeof(uint32_t) * static_cast<size_t>(T) * nb, s));
        }
        TM_CUDA(cudaMemsetAsync(L.counters.p, 0, 4 * sizeof(uint32_t), s));
        uint32_t *d_cand_count = L.counters.as<uint32_t>();
        uint32_t *d_list_count = d_cand_count + 1;
        tmb::ScanArgs a{};
        a.x = ctx->clean.as<float>();
        a.q = g.q.as<float>();
        a.tp = g.tp.as<TemplParam>();
        a.w0 = w0;
        a.W = static_cast<uint32_t>(W);
        a.m_pad = g.k_stride;
        a.T = T;
        a.bmin_u = L.bmin_u.as<uint32_t>();
        a.bmin_l = L.bmin_l.as<uint32_t>();
        a.nb = nb;
        a.cand = L.cand.as<Candidate>();
        a.cand_count = d_cand_count;
        a.cand_cap = L.cand_cap;
        a.q_hi = g.q_hi.p;
        a.q_lo = g.q_lo.p;
        a.t_rows = g.t_rows;
        a.err = reinterpret_cast<int *>(d_cand_count + 2);
        a.raw = ctx->raw.as<float>();
        a.P = ctx->prefix.as<double2>();
        a.PT = ctx->ptot.as<double2>();
        a.PC = ctx->pcen.as<double>();
        a.run = ctx->run.as<uint16_t>();
        a.tiles = g.d_tiles.as<tmb::TileInfo>();
        a.k_stride = g.k_stride;
        a.n = ctx->n;
        if (L.profile)
            TM_CUDA(cudaEventRecord(L.ev0, s));
        a.col_tile = g.col_tile;
        if (g.fft)
            fft_contract(ctx, L, g, a);
        else
        {
            TM_CUDA(g.col_tile > 0 ? tmb::launch_scan_wm(a, s) : tmb::launch_scan_umma(a, s));
            count_launch(L);
        }
        if (L.profile)
        {
            TM_CUDA(cudaEventRecord(L.ev1, s));
            TM_CUDA(cudaEventSynchronize(L.ev1));
            float ms = 0.0f;
            TM_CUDA(cudaEventElapsedTime(&ms, L.ev0, L.ev1));
            L.kname = g.fft ? "fft" : (g.col_tile > 0 ? "k_scan_wm" : "k_scan_umma");
            L.prof_launches++;
            L.prof_ms += ms;
            L.phase_ms[0] += ms;
            L.prof_flops += flops;
        }
        if (nk > 0)
        {
            TM_CUDA(tmb::launch_bucket_select(L.bmin_u.as<uint32_t>(), nb, g.tp.as<TemplParam>(),
                                              g.slots.as<int>(), nk, L.tkey.as<uint32_t>(), s));
            for (int la = 0; la < 3; la++)
            {
                L.list.reserve(sizeof(uint2) * static_cast<size_t>(L.list_cap));
                TM_CUDA(cudaMemsetAsync(d_list_count, 0, sizeof(uint32_t), s));
                TM_CUDA(tmb::launch_list_buckets(L.bmin_l.as<uint32_t>(), nb, g.slots.as<int>(), nk,
                                                 L.tkey.as<uint32_t>(), L.list.as<uint2>(), d_list_count,
                                                 L.list_cap, s));
                TM_CUDA(cudaMemcpyAsync(hc + 1, d_list_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
                TM_CUDA(cudaStreamSynchronize(s));
                count_launch(L, 2);
                if (hc[1] <= L.list_cap)
                    break;
                L.list_cap = hc[1] + hc[1] / 2;
            }
            if (hc[1] > L.list_cap)
                throw Failure{TM_ERR_NO_MEMORY, "bucket list overflow"};
            TM_CUDA(tmb::launch_passb_mixed(L.list.as<uint2>(), hc[1], ctx->clean.as<float>(),
                                            ctx->raw.as<float>(), ctx->prefix.as<double2>(), ctx->ptot.as<double2>(),
                                            ctx->pcen.as<double>(), ctx->run.as<uint16_t>(), g.q.as<float>(),
                                            g.tp.as<TemplParam>(),
                                            L.tkey.as<uint32_t>(), w0, L.cand.as<Candidate>(), d_cand_count,
                                            L.cand_cap, s));
            if (hc[1] > 0)
                count_launch(L);
        }
        if (L.profile)
            TM_CUDA(cudaEventRecord(L.ev2, s));
        TM_CUDA(cudaMemcpyAsync(hc, d_cand_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        TM_CUDA(cudaMemcpyAsync(hc + 2, d_cand_count + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        TM_CUDA(cudaStreamSynchronize(s));
        if (L.profile)
            add_span(L, 1, L.ev1, L.ev2);
        if (hc[2] != 0)
            throw Failure{TM_ERR_TIMEOUT, "contraction kernel gave up waiting (code " + std::to_string(hc[2]) + ")"};
        ncand = hc[0];
        if (ncand <= L.cand_cap)
            break;
        L.cand_cap = ncand + ncand / 2;
        if (attempt == 2)
            throw Failure{TM_ERR_NO_MEMORY, "candidate buffer overflow"};
    }
    std::vector<uint16_t> run;
    std::vector<float> raw;
    rescore_and_answer(ctx, L, g, ncand, w0, res, [&](int t, std::vector<Hit> &degenerate) {
        if (run.empty())
        {
            run.resize(W);
            raw.resize(W);
            TM_CUDA(cudaMemcpy(run.data(), ctx->run.as<uint16_t>() + w0, W * sizeof(uint16_t), cudaMemcpyDeviceToHost));
            TM_CUDA(cudaMemcpy(raw.data(), ctx->raw.as<float>() + w0, W * sizeof(float), cudaMemcpyDeviceToHost));
        }
        const TemplParam &p = g.htp[t];
        for (uint64_t j = 0; j < p.wcount; j++)
            if (run[j] >= p.m && raw[j] != TM_MISSING_VALUE)
                degenerate.push_back(Hit{w0 + j, FLT_MAX});
    });
}

// Modelled milliseconds of 128 template rows x 2^25 windows of shape v at K samples:
// linear between the measured K, proportional to K above the largest, flat below the
// smallest (epilogue-bound there).
double tile_time(const tm_ctx *ctx, bool mixed, int v, double k)
{
    static const double ks[4] = {256.0, 1024.0, 4096.0, 16384.0};
    const double *t = ctx->tile_ms[mixed ? 1 : 0][v];
    if (k <= ks[0])
        return t[0];
    if (k >= ks[3])
        return t[3] * k / ks[3];
    int i = 0;
    while (k > ks[i + 1])
        i++;
    return t[i] + (t[i + 1] - t[i]) * (k - ks[i]) / (ks[i + 1] - ks[i]);
}

// Tile shape of a group: 0 (row tiles of 128 templates, k_scan_umma) or the column-tile
// size (k_scan_wm). Each shape's modelled time sums its tiles (consecutive in length
// order; a tile costs its rows at its longest template's K); the least wins. *cost gets
// the winner's modelled milliseconds per 2^25 windows.
int plan_col_tile(const tm_ctx *ctx, const tm_request *reqs, const std::vector<int> &idx, double *cost = nullptr)
{
    std::vector<int> m(idx.size());
    for (size_t i = 0; i < idx.size(); i++)
        m[i] = reqs[idx[i]].m;
    std::sort(m.begin(), m.end(), std::greater<int>());
    const bool mixed = !m.empty() && m.front() != m.back();
    const int shapes[4] = {128, 128, 64, 32};
    double costs[4];
    for (int v = 0; v < 4; v++)
    {
        const size_t rows = static_cast<size_t>(shapes[v]);
        costs[v] = 0.0;
        for (size_t i = 0; i < m.size(); i += rows) // row tiles may close early (65 lengths): ignored
            costs[v] += static_cast<double>(rows) / 128.0 *
                        tile_time(ctx, mixed, v, static_cast<double>((m[i] + 63) & ~63));
    }
    int v = 0;
    switch (ctx->tiles)
    {
    case TM_TILES_ROWS:
        v = 0;
        break;
    case TM_TILES_COLS_128:
        v = 1;
        break;
    case TM_TILES_COLS_64:
        v = 2;
        break;
    case TM_TILES_COLS_32:
        v = 3;
        break;
    default:
        for (int u = 1; u < 4; u++)
            if (costs[u] < costs[v])
                v = u;
    }
    if (cost)
        *cost = costs[v];
    return v == 0 ? 0 : shapes[v];
}

// Modelled milliseconds per 2^25 windows of templates with lengths m[0..n) (sorted,
// longest first) in the tile shape TM_TILES_AUTO would pick (or the forced one).
double tensor_cost_sorted(const tm_ctx *ctx, const int *m, size_t n)
{
    if (n == 0)
        return 0.0;
    const bool mixed = m[0] != m[n - 1];
    const int shapes[4] = {128, 128, 64, 32};
    double best = 0.0;
    for (int v = 0; v < 4; v++)
    {
        if ((ctx->tiles == TM_TILES_ROWS && v != 0) || (ctx->tiles == TM_TILES_COLS_128 && v != 1) ||
            (ctx->tiles == TM_TILES_COLS_64 && v != 2) || (ctx->tiles == TM_TILES_COLS_32 && v != 3))
            continue;
        double c = 0.0;
        for (size_t i = 0; i < n; i += static_cast<size_t>(shapes[v]))
            c += shapes[v] / 128.0 * tile_time(ctx, mixed, v, static_cast<double>((m[i] + 63) & ~63));
        if (best == 0.0 || c < best)
            best = c;
    }
    return best;
}

// How many of a group's templates (ordered longest first) go to the FFT branch: all of
// them when it is forced (TM_TILES_FFT); under TM_TILES_AUTO with the automatic kernel,
// the f minimising f x (the FFT's per-template time) + the tensor cost of the other
// templates: the longest templates set a tile's K extent, so moving a few of them to the
// FFT (whose cost does not grow with the length) can shorten every tile they would have
// padded. Lengths up to 16384 (the FFT pieces' step); otherwise none.
size_t plan_fft_split(const tm_ctx *ctx, const tm_request *reqs, const std::vector<int> &sorted_idx)
{
    const size_t n = sorted_idx.size();
    if (n == 0 || ctx->kernel == TM_KERNEL_FP32 || !tmb::umma_supported(0, 0, 0))
        return 0;
    for (int i : sorted_idx)
        if (reqs[i].m > tmb::kFftS)
            return 0;
    if (ctx->tiles == TM_TILES_FFT)
        return n;
    if (ctx->tiles != TM_TILES_AUTO || ctx->kernel != TM_KERNEL_AUTO)
        return 0;
    std::vector<int> m(n);
    for (size_t i = 0; i < n; i++)
        m[i] = reqs[sorted_idx[i]].m;
    size_t best_f = 0;
    double best = tensor_cost_sorted(ctx, m.data(), n);
    for (size_t f = 1; f <= n; f++)
    {
        const double c = static_cast<double>(f) * ctx->fft_ms + tensor_cost_sorted(ctx, m.data() + f, n - f);
        if (c < best)
        {
            best = c;
            best_f = f;
        }
    }
    return best_f;
}

// Groups of a batch. Lengths with a full 128-template tile (or any length, on the FP32
// kernel) get their own group with per-length statistics; the remaining templates of
// several lengths share one mixed-length group on the tensor cores.
void create_batch(tm_ctx *ctx, Lane &L, const tm_request *requests, int count, tm_batch &b, bool serving = false)
{
    b.count = count;
    const bool tensor = ctx->kernel != TM_KERNEL_FP32 && tmb::umma_supported(0, 0, 0);
    // candidate groups (lists of requests); each is then split between the FFT branch and
    // the contraction (plan_fft_split)
    std::vector<std::vector<int>> lists;
    if (serving) // one list over the resident prefix sums, whatever the lengths
    {
        lists.emplace_back(static_cast<size_t>(count));
        for (int i = 0; i < count; i++)
            lists[0][i] = i;
    }
    else
    {
        std::map<int, std::vector<int>> by_m;
        for (int i = 0; i < count; i++)
            by_m[requests[i].m].push_back(i);
        std::vector<int> rest;
        for (auto &kv : by_m)
        {
            if (!tensor || kv.second.size() >= 128 || kv.first > 16384)
                lists.push_back(kv.second);
            else
                rest.insert(rest.end(), kv.second.begin(), kv.second.end());
        }
        if (!rest.empty())
            lists.push_back(rest);
    }
    struct Spec
    {
        std::vector<int> idx;
        int kind; // 0: one length, per-length statistics; 1: prefix statistics, tiles; 2: FFT branch
    };
    std::vector<Spec> specs;
    for (std::vector<int> &list : lists)
    {
        std::stable_sort(list.begin(), list.end(), [&](int a, int c) { return requests[a].m > requests[c].m; });
        const size_t f = tensor ? plan_fft_split(ctx, requests, list) : 0;
        if (f > 0)
            specs.push_back(Spec{std::vector<int>(list.begin(), list.begin() + f), 2});
        if (f < list.size())
        {
            std::vector<int> part(list.begin() + f, list.end());
            const bool one_length = requests[part.front()].m == requests[part.back()].m;
            specs.push_back(Spec{part, one_length && !serving ? 0 : 1});
        }
    }
    b.groups.resize(specs.size());
    for (size_t gi = 0; gi < specs.size(); gi++)
    {
        GroupPlan &g = b.groups[gi];
        const std::vector<int> &idx = specs[gi].idx;
        const int m = requests[idx.front()].m;
        if (specs[gi].kind == 2)
        {
            prepare_group_mixed(ctx, L, idx, requests, g, b.h2d_bytes, 0);
            g.fft = true;
        }
        else if (specs[gi].kind == 0)
            prepare_group(ctx, L, m, idx, requests, g, b.h2d_bytes,
                          tensor && m <= 16384 ? plan_col_tile(ctx, requests, idx) : 0);
        else
            prepare_group_mixed(ctx, L, idx, requests, g, b.h2d_bytes, plan_col_tile(ctx, requests, idx));
    }
}

void run_batch(tm_ctx *ctx, Lane &L, tm_batch &b, tm_result &res)
{
    res.answers.assign(static_cast<size_t>(b.count), Answer());
    res.blocks.clear();
    L.last_candidates = 0;
    for (GroupPlan &g : b.groups)
    {
        if (g.mixed)
            execute_group_mixed(ctx, L, g, res);
        else
            execute_group(ctx, L, g, res);
    }
}

int validate_requests(const tm_ctx *ctx, const tm_request *reqs, int count)
{
    if (count < 0 || (count > 0 && reqs == nullptr))
        return TM_ERR_ARGUMENT;
    for (int i = 0; i < count; i++)
    {
        const tm_request &r = reqs[i];
        if (r.templ == nullptr || r.m < 1 || static_cast<uint64_t>(r.m) > ctx->n || r.merge_offset < 0)
            return TM_ERR_ARGUMENT;
        if (r.mode == TM_MODE_KNN)
        {
            if (r.k < 1)
                return TM_ERR_ARGUMENT;
        }
        else if (r.mode != TM_MODE_THRESHOLD)
            return TM_ERR_ARGUMENT;
    }
    return TM_OK;
}

} // namespace


// ---- serving: continuous batching over the resident waveform ------------------------
//
// Requests are submitted one at a time from any thread and queue in arrival order.
// Each worker owns a lane (stream + scratch) and loops: it admits the oldest pending
// requests, as many as max_batch and the device-memory budget for requests in flight
// allow (a request larger than the whole budget still runs, alone), prepares them as
// one mixed-length group over the resident prefix sums, runs it and completes every
// request of it. While one worker's batch is on the GPU, the others admit what arrived
// meanwhile and prepare, launch or finish theirs, so batches overlap on the device and
// with the host work around them. A request's answers are those of the same request
// run alone: each (template, window) pair is scored, rescored and selected by itself.

struct ServeItem
{
    uint64_t ticket = 0;
    std::vector<float> templ; // owned copy
    tm_request req{};
    uint64_t bytes = 0; // admission estimate
    double submit_ms = 0.0;
};

struct Server
{
    tm_ctx *ctx = nullptr;
    tm_serve_config cfg{};
    std::vector<std::unique_ptr<Lane>> lanes;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable work_cv, done_cv;
    std::deque<ServeItem> pending;
    std::deque<tm_completion> done;
    uint64_t next_ticket = 1, in_flight_bytes = 0, in_flight = 0, launches = 0;
    bool stopping = false, stopped = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now_ms() const
    {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    ~Server()
    {
        for (tm_completion &c : done)
            delete c.result;
    }
};

// Device bytes a request holds while in flight: its template row (FP32, two BF16 halves,
// block order) at up to the longest length a batch can have, plus its share of the
// candidate, sort and answer buffers: kNN about 2k-1 buckets of windows, threshold a
// fixed fraction of the windows (an estimate: the buffers grow when a batch needs more).
static uint64_t serve_bytes(const tm_ctx *ctx, const tm_request &r)
{
    const uint64_t W = ctx->n - static_cast<uint64_t>(r.m) + 1;
    const uint64_t row = 10ull * 16384 + sizeof(TemplParam);
    const uint64_t cands = r.mode == TM_MODE_KNN ? std::min<uint64_t>(W, (2ull * r.k) * tmb::kBucket / 4)
                                                 : std::max<uint64_t>(W / 512, 1024);
    return row + 48ull * cands;
}

// Admission (under the server's lock). A batch is built a tile at a time: the 128 rows of
// a contraction tile share one K extent, their longest template, so rows not longer than
// that cost nothing extra. Each tile opens with the oldest pending request (so every batch
// admits the oldest, and later arrivals never hold a request back indefinitely) and fills
// with the longest pending requests not longer than it; with a long queue the tiles hold
// similar lengths.
// Stops at max_batch or at the memory budget (a first request alone is always admitted).
static void admit(Server *sv, std::vector<ServeItem> &batch, uint64_t &bytes)
{
    auto fits = [&](uint64_t b) {
        return (sv->in_flight_bytes == 0 && batch.empty()) || sv->in_flight_bytes + bytes + b <= sv->cfg.memory_budget;
    };
    std::vector<size_t> order;
    std::vector<char> chosen;
    while (!sv->pending.empty() && static_cast<int>(batch.size()) < sv->cfg.max_batch)
    {
        if (!fits(sv->pending.front().bytes))
            return;
        const int cap_m = sv->pending.front().req.m;
        bytes += sv->pending.front().bytes;
        batch.push_back(std::move(sv->pending.front()));
        sv->pending.pop_front();
        const size_t room = std::min<size_t>(127, static_cast<size_t>(sv->cfg.max_batch) - batch.size());
        order.clear();
        for (size_t i = 0; i < sv->pending.size(); i++)
            if (sv->pending[i].req.m <= cap_m)
                order.push_back(i);
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t x, size_t y) { return sv->pending[x].req.m > sv->pending[y].req.m; });
        chosen.assign(sv->pending.size(), 0);
        size_t taken = 0;
        for (size_t i : order)
        {
            if (taken == room || !fits(sv->pending[i].bytes))
                break;
            bytes += sv->pending[i].bytes;
            batch.push_back(std::move(sv->pending[i]));
            chosen[i] = 1;
            taken++;
        }
        if (taken > 0)
        {
            std::deque<ServeItem> rest;
            for (size_t i = 0; i < sv->pending.size(); i++)
                if (!chosen[i])
                    rest.push_back(std::move(sv->pending[i]));
            sv->pending.swap(rest);
        }
    }
}

static void serve_worker(Server *sv, Lane *L)
{
    tm_ctx *ctx = sv->ctx;
    cudaSetDevice(ctx->device);
    // one batch object per worker, its device buffers grown and reused: freeing device
    // memory would wait for the other lanes' kernels
    tm_batch b;
    for (;;)
    {
        std::vector<ServeItem> batch;
        uint64_t bytes = 0;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            for (;;)
            {
                if (sv->pending.empty() && sv->stopping)
                    return;
                admit(sv, batch, bytes);
                if (!batch.empty())
                    break;
                sv->work_cv.wait(lk); // nothing pending, or the budget is full: wait for either to change
            }
            sv->in_flight_bytes += bytes;
            sv->in_flight += batch.size();
        }
        const double start = sv->now_ms();
        std::vector<tm_request> reqs(batch.size());
        for (size_t i = 0; i < batch.size(); i++)
        {
            reqs[i] = batch[i].req;
            reqs[i].templ = batch[i].templ.data();
        }
        auto res = std::make_unique<tm_result>();
        int code = TM_OK;
        std::string what;
        try
        {
            b.h2d_bytes = 0;
            create_batch(ctx, *L, reqs.data(), static_cast<int>(reqs.size()), b, true);
            run_batch(ctx, *L, b, *res);
        }
        catch (const Failure &f)
        {
            code = f.code;
            what = f.what;
        }
        catch (const std::bad_alloc &)
        {
            code = TM_ERR_NO_MEMORY;
        }
        catch (const std::exception &e)
        {
            code = TM_ERR_STATE;
            what = e.what();
        }
        const double end = sv->now_ms();
        std::vector<tm_completion> out(batch.size());
        for (size_t i = 0; i < batch.size(); i++)
        {
            tm_completion &c = out[i];
            c.ticket = batch[i].ticket;
            c.status = code;
            c.result = nullptr;
            c.submit_ms = batch[i].submit_ms;
            c.start_ms = start;
            c.done_ms = end;
            c.batch_size = static_cast<int>(batch.size());
            if (code == TM_OK)
            {
                // one result per request, sharing the batch's pinned answer blocks
                auto r = std::make_unique<tm_result>();
                r->answers.push_back(std::move(res->answers[i]));
                r->blocks = res->blocks;
                c.result = r.release();
            }
        }
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->in_flight_bytes -= bytes;
            sv->in_flight -= batch.size();
            sv->launches += static_cast<uint64_t>(L->all_launches);
            L->all_launches = 0;
            for (tm_completion &c : out)
                sv->done.push_back(c);
        }
        sv->done_cv.notify_all();
        sv->work_cv.notify_all();
    }
}

// Completes what was submitted, then joins the workers; completions stay pollable.
static void stop_server(tm_ctx *ctx)
{
    Server *sv = ctx->server.get();
    if (sv == nullptr || sv->stopped)
        return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stopping = true;
    }
    sv->work_cv.notify_all();
    for (std::thread &t : sv->threads)
        t.join();
    sv->threads.clear();
    for (auto &L : sv->lanes)
        L->close();
    sv->lanes.clear();
    sv->stopped = true;
}

// tm_bound_diagnostics for the window-major kernel or the FFT branch: the templates (all of
// length m) as one group in column tiles of the context's shape (or through the FFT
// branch), statistics from the prefix sums.
static void bound_diagnostics_wm(tm_ctx *ctx, int m, const std::vector<int> &idx, const std::vector<tm_request> &reqs,
                                 float *d, float *e, float *exact)
{
    Lane &L = ctx->main;
    cudaStream_t s = L.stream;
    const int count = static_cast<int>(idx.size());
    ensure_prefix(ctx, L);
    GroupPlan g;
    uint64_t h2d = 0;
    prepare_group_mixed(ctx, L, idx, reqs.data(), g, h2d, plan_col_tile(ctx, reqs.data(), idx));
    const uint64_t W = g.w_max;
    if (W == 0 || W * static_cast<uint64_t>(count) > (1ull << 31))
        throw Failure{TM_ERR_ARGUMENT, "diagnostics need 0 < windows x templates <= 2^31"};
    for (int t = 0; t < g.T; t++)
        g.htp[t].thr_ed = -FLT_MAX; // emit nothing
    TM_CUDA(cudaMemcpyAsync(g.tp.p, g.htp.data(), sizeof(TemplParam) * g.T, cudaMemcpyHostToDevice, s));
    const size_t pairs = W * static_cast<size_t>(count);
    DevBuf dd, de, dc, dx;
    dd.reserve(pairs * sizeof(float));
    de.reserve(pairs * sizeof(float));
    L.counters.reserve(8 * sizeof(uint32_t));
    TM_CUDA(cudaMemsetAsync(L.counters.p, 0, 8 * sizeof(uint32_t), s));
    TM_CUDA(cudaMemsetAsync(dd.p, 0xff, pairs * sizeof(float), s)); // NaN where nothing was written
    TM_CUDA(cudaMemsetAsync(de.p, 0xff, pairs * sizeof(float), s));
    L.cand.reserve(sizeof(Candidate) * 16);
    const uint32_t nb = static_cast<uint32_t>((W + tmb::kBucket - 1) / tmb::kBucket);
    L.bmin_u.reserve(sizeof(uint32_t) * static_cast<size_t>(g.T) * nb);
    L.bmin_l.reserve(sizeof(uint32_t) * static_cast<size_t>(g.T) * nb);
    tmb::ScanArgs a{};
    a.x = ctx->clean.as<float>();
    a.q = g.q.as<float>();
    a.tp = g.tp.as<TemplParam>();
    a.w0 = ctx->range_first;
    a.W = static_cast<uint32_t>(W);
    a.T = g.T;
    a.bmin_u = L.bmin_u.as<uint32_t>();
    a.bmin_l = L.bmin_l.as<uint32_t>();
    a.nb = nb;
    a.cand = L.cand.as<Candidate>();
    a.cand_count = L.counters.as<uint32_t>();
    a.cand_cap = 0;
    a.q_hi = g.q_hi.p;
    a.q_lo = g.q_lo.p;
    a.t_rows = g.t_rows;
    a.err = reinterpret_cast<int *>(L.counters.as<uint32_t>() + 2);
    a.dbg_d = dd.as<float>();
    a.dbg_e = de.as<float>();
    a.raw = ctx->raw.as<float>();
    a.P = ctx->prefix.as<double2>();
    a.PT = ctx->ptot.as<double2>();
    a.PC = ctx->pcen.as<double>();
    a.run = ctx->run.as<uint16_t>();
    a.tiles = g.d_tiles.as<tmb::TileInfo>();
    a.k_stride = g.k_stride;
    a.n = ctx->n;
    a.col_tile = g.col_tile;
    if (ctx->tiles == TM_TILES_FFT)
        fft_contract(ctx, L, g, a);
    else
    {
        TM_CUDA(g.col_tile > 0 ? tmb::launch_scan_wm(a, s) : tmb::launch_scan_umma(a, s));
        count_launch(L);
    }
    TM_CUDA(cudaMemcpyAsync(d, dd.p, pairs * sizeof(float), cudaMemcpyDeviceToHost, s));
    TM_CUDA(cudaMemcpyAsync(e, de.p, pairs * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (exact != nullptr)
    {
        std::vector<Candidate> all(pairs);
        for (int t = 0; t < count; t++)
            for (uint64_t j = 0; j < W; j++)
                all[static_cast<size_t>(t) * W + j] = Candidate{static_cast<uint32_t>(t), static_cast<uint32_t>(j)};
        dc.reserve(pairs * sizeof(Candidate));
        dx.reserve(pairs * sizeof(float));
        TM_CUDA(cudaMemcpyAsync(dc.p, all.data(), pairs * sizeof(Candidate), cudaMemcpyHostToDevice, s));
        TM_CUDA(tmb::launch_rescore(dc.as<Candidate>(), static_cast<uint32_t>(pairs), g.tp.as<TemplParam>(),
                                    g.q.as<float>(), g.order.as<int>(), ctx->raw.as<float>(), ctx->range_first,
                                    dx.as<float>(), s));
        count_launch(L);
        TM_CUDA(cudaMemcpyAsync(exact, dx.p, pairs * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    uint32_t err = 0;
    TM_CUDA(cudaMemcpyAsync(&err, L.counters.as<uint32_t>() + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    TM_CUDA(cudaStreamSynchronize(s));
    g.release();
    if (err != 0)
        throw Failure{TM_ERR_TIMEOUT, "contraction kernel gave up waiting"};
}

// ---------------------------------------------------------------------------------
extern "C" {

int tm_ctx_create(const float *raw, uint64_t n, int device, tm_ctx **out)
{
    if (out == nullptr || raw == nullptr || n == 0)
        return TM_ERR_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return TM_ERR_NO_DEVICE;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10)
        return TM_ERR_NO_DEVICE;
    auto ctx = std::make_unique<tm_ctx>();
    ctx->device = device;
    ctx->n = n;
    const int rc = guarded(ctx.get(), [&] {
        TM_CUDA(cudaSetDevice(device));
        ctx->main.open();
        const uint64_t total = n + tmb::kStagePad;
        ctx->raw.reserve(sizeof(float) * total);
        ctx->clean.reserve(sizeof(float) * total);
        TM_CUDA(cudaMemsetAsync(ctx->raw.p, 0, sizeof(float) * total, ctx->main.stream));
        TM_CUDA(cudaMemcpyAsync(ctx->raw.p, raw, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->main.stream));
        TM_CUDA(tmb::launch_clean(ctx->raw.as<float>(), ctx->clean.as<float>(), n, total, ctx->main.stream));
        TM_CUDA(cudaStreamSynchronize(ctx->main.stream));
    });
    if (rc != TM_OK)
    {
        tm_ctx_destroy(ctx.release());
        return rc;
    }
    *out = ctx.release();
    return TM_OK;
}

int tm_ctx_destroy(tm_ctx *ctx)
{
    if (ctx == nullptr)
        return TM_OK;
    cudaSetDevice(ctx->device);
    stop_server(ctx);
    ctx->main.close();
    for (auto &kv : ctx->lengths)
    {
        kv.second->mean.release();
        kv.second->inv.release();
        kv.second->flags.release();
    }
    for (DevBuf *b : {&ctx->prefix, &ctx->ptot, &ctx->pcen, &ctx->run, &ctx->raw, &ctx->clean, &ctx->suf,
                      &ctx->fft_X, &ctx->fft_shift, &ctx->fft_norm})
        b->release();
    delete ctx;
    return TM_OK;
}

const char *tm_last_error(const tm_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int tm_set_kernel(tm_ctx *ctx, int kernel)
{
    if (ctx == nullptr || kernel < TM_KERNEL_AUTO || kernel > TM_KERNEL_SPLIT_BF16)
        return TM_ERR_ARGUMENT;
    if (ctx->server && !ctx->server->stopped)
        return TM_ERR_STATE;
    ctx->kernel = kernel;
    return TM_OK;
}

int tm_set_tiles(tm_ctx *ctx, int tiles)
{
    if (ctx == nullptr || tiles < TM_TILES_AUTO || tiles > TM_TILES_FFT)
        return TM_ERR_ARGUMENT;
    ctx->tiles = tiles;
    return TM_OK;
}

int tm_autotune(tm_ctx *ctx, double *ms, int capacity)
{
    if (ctx == nullptr || capacity < 0 || (capacity > 0 && ms == nullptr))
        return TM_ERR_ARGUMENT;
    const int rc = guarded(ctx, [&] {
        TM_CUDA(cudaSetDevice(ctx->device));
        if (ctx->kernel == TM_KERNEL_FP32 || !tmb::umma_supported(0, 0, 0))
            throw Failure{TM_ERR_STATE, "the tile shapes are those of the tensor-core kernel"};
        // a synthetic record: a random walk of small steps plus noise (xorshift)
        const uint64_t n = 1ull << 23;
        std::vector<float> x(n);
        uint64_t st = 0x9E3779B97F4A7C15ull;
        auto rnd = [&] {
            st ^= st << 13;
            st ^= st >> 7;
            st ^= st << 17;
            return static_cast<float>((st >> 40) * (1.0 / 16777216.0)) - 0.5f;
        };
        float level = 0.0f;
        for (uint64_t i = 0; i < n; i++)
        {
            level = 0.95f * level + rnd();
            x[i] = level + 0.1f * rnd();
        }
        tm_ctx *tc = nullptr;
        const int rc = tm_ctx_create(x.data(), n, ctx->device, &tc);
        if (rc != TM_OK)
            throw Failure{rc, "autotune context"};
        std::unique_ptr<tm_ctx, int (*)(tm_ctx *)> hold(tc, tm_ctx_destroy);
        const int ks[4] = {256, 1024, 4096, 16384};
        std::vector<std::vector<float>> temps(128);
        std::vector<tm_request> reqs(128);
        double table[2][4][4];
        for (int mixed = 0; mixed < 2; mixed++)
            for (int ki = 0; ki < 4; ki++)
            {
                for (int t = 0; t < 128; t++)
                {
                    const int m = ks[ki] - (mixed && (t & 1) ? 16 : 0);
                    temps[t].resize(static_cast<size_t>(m));
                    for (int i = 0; i < m; i++)
                        temps[t][i] = std::sin(0.003f * static_cast<float>(i) * (1.0f + 0.01f * t) +
                                               1e-6f * static_cast<float>(i) * static_cast<float>(i));
                    reqs[t] = tm_request{temps[t].data(), m, TM_MODE_THRESHOLD, 1, 0, 0.995f, 0u};
                }
                const double windows = static_cast<double>(n - static_cast<uint64_t>(ks[ki]) + 1);
                for (int v = 0; v < 4; v++)
                {
                    tc->tiles = TM_TILES_ROWS + v;
                    tm_batch b;
                    create_batch(tc, tc->main, reqs.data(), 128, b);
                    tm_result res;
                    run_batch(tc, tc->main, b, res); // warm-up
                    tc->main.profile = true;
                    tc->main.prof_ms = 0.0;
                    tc->main.prof_launches = 0;
                    for (int r = 0; r < 2; r++)
                        run_batch(tc, tc->main, b, res);
                    tc->main.profile = false;
                    const double per = tc->main.prof_ms / std::max<int64_t>(tc->main.prof_launches, 1);
                    table[mixed][v][ki] = per * (33554432.0 / windows);
                }
            }
        // the FFT branch: 8 of the last templates (its time does not depend on the length)
        tc->tiles = TM_TILES_FFT;
        {
            tm_batch b;
            create_batch(tc, tc->main, reqs.data(), 8, b);
            tm_result res;
            run_batch(tc, tc->main, b, res);
            tc->main.profile = true;
            tc->main.prof_ms = 0.0;
            tc->main.prof_launches = 0;
            run_batch(tc, tc->main, b, res);
            tc->main.profile = false;
        }
        const double fft_ms = tc->main.prof_ms / 8.0 * (33554432.0 / static_cast<double>(n));
        std::memcpy(ctx->tile_ms, table, sizeof(table));
        ctx->fft_ms = fft_ms;
        for (int i = 0; i < std::min(capacity, 33); i++)
            ms[i] = i < 32 ? (&table[0][0][0])[i] : fft_ms;
    });
    return rc == TM_OK ? 33 : rc;
}

int tm_set_tile_model(tm_ctx *ctx, const double *ms, int count)
{
    if (ctx == nullptr || ms == nullptr || (count != 32 && count != 33))
        return TM_ERR_ARGUMENT;
    for (int i = 0; i < count; i++)
        if (!(ms[i] > 0.0) || !std::isfinite(ms[i]))
            return TM_ERR_ARGUMENT;
    std::memcpy(ctx->tile_ms, ms, sizeof(ctx->tile_ms));
    if (count == 33)
        ctx->fft_ms = ms[32];
    return TM_OK;
}

int tm_set_window_range(tm_ctx *ctx, uint64_t first, uint64_t count)
{
    if (ctx == nullptr || count == 0)
        return TM_ERR_ARGUMENT;
    if (ctx->server && !ctx->server->stopped)
        return TM_ERR_STATE;
    return guarded(ctx, [&] {
        TM_CUDA(cudaSetDevice(ctx->device));
        TM_CUDA(cudaStreamSynchronize(ctx->main.stream));
        for (auto &kv : ctx->lengths)
        {
            kv.second->mean.release();
            kv.second->inv.release();
            kv.second->flags.release();
        }
        ctx->lengths.clear();
        ctx->range_first = first;
        ctx->range_count = count;
    });
}

int tm_prepare_length(tm_ctx *ctx, int m)
{
    if (ctx == nullptr || m < 1 || static_cast<uint64_t>(m) > ctx->n)
        return TM_ERR_ARGUMENT;
    return guarded(ctx, [&] {
        TM_CUDA(cudaSetDevice(ctx->device));
        ensure_length(ctx, ctx->main, m);
        TM_CUDA(cudaStreamSynchronize(ctx->main.stream));
    });
}

int tm_window_stats(tm_ctx *ctx, int m, uint64_t first, uint64_t count, float *mean, float *stddev)
{
    if (ctx == nullptr || m < 1 || static_cast<uint64_t>(m) > ctx->n || mean == nullptr || stddev == nullptr)
        return TM_ERR_ARGUMENT;
    const uint64_t total = ctx->n - static_cast<uint64_t>(m) + 1;
    if (first > total || count > total - first)
        return TM_ERR_ARGUMENT;
    if (count == 0)
        return TM_OK;
    return guarded(ctx, [&] {
        TM_CUDA(cudaSetDevice(ctx->device));
        DevBuf dm, ds;
        dm.reserve(count * sizeof(float));
        ds.reserve(count * sizeof(float));
        TM_CUDA(tmb::launch_reference_stats(ctx->raw.as<float>(), m, first, count, dm.as<float>(), ds.as<float>(),
                                           ctx->main.stream));
        count_launch(ctx->main);
        TM_CUDA(cudaMemcpyAsync(mean, dm.p, count * sizeof(float), cudaMemcpyDeviceToHost, ctx->main.stream));
        TM_CUDA(cudaMemcpyAsync(stddev, ds.p, count * sizeof(float), cudaMemcpyDeviceToHost, ctx->main.stream));
        TM_CUDA(cudaStreamSynchronize(ctx->main.stream));
        dm.release();
        ds.release();
    });
}

int tm_batch_create(tm_ctx *ctx, const tm_request *requests, int count, tm_batch **out)
{
    if (ctx == nullptr || out == nullptr)
        return TM_ERR_ARGUMENT;
    *out = nullptr;
    const int v = validate_requests(ctx, requests, count);
    if (v != TM_OK)
    {
        ctx->err = "invalid request";
        return v;
    }
    auto b = std::make_unique<tm_batch>();
    const int rc = guarded(ctx, [&] {
        TM_CUDA(cudaSetDevice(ctx->device));
        create_batch(ctx, ctx->main, requests, count, *b);
    });
    if (rc == TM_OK)
        *out = b.release();
    return rc;
}

int tm_batch_run(tm_ctx *ctx, tm_batch *batch, tm_result **out)
{
    if (ctx == nullptr || batch == nullptr || out == nullptr)
        return TM_ERR_ARGUMENT;
    *out = nullptr;
    auto res = std::make_unique<tm_result>();
    const int rc = guarded(ctx, [&] {
        TM_CUDA(cudaSetDevice(ctx->device));
        run_batch(ctx, ctx->main, *batch, *res);
    });
    if (rc == TM_OK)
        *out = res.release();
    return rc;
}

int tm_batch_destroy(tm_batch *batch)
{
    delete batch;
    return TM_OK;
}

int tm_batch_h2d_bytes(const tm_batch *batch, uint64_t *bytes)
{
    if (batch == nullptr || bytes == nullptr)
        return TM_ERR_ARGUMENT;
    *bytes = batch->h2d_bytes;
    return TM_OK;
}

int tm_scan_batch(tm_ctx *ctx, const tm_request *requests, int count, tm_result **out)
{
    tm_batch *b = nullptr;
    int rc = tm_batch_create(ctx, requests, count, &b);
    if (rc != TM_OK)
        return rc;
    rc = tm_batch_run(ctx, b, out);
    tm_batch_destroy(b);
    return rc;
}

int tm_search_knn(tm_ctx *ctx, const float *queries, int count, int m, int k, int merge_offset, uint64_t *I, float *D)
{
    if (ctx == nullptr || queries == nullptr || I == nullptr || D == nullptr || count < 0 || k < 1)
        return TM_ERR_ARGUMENT;
    std::vector<tm_request> reqs(static_cast<size_t>(count));
    for (int i = 0; i < count; i++)
        reqs[i] = tm_request{queries + static_cast<size_t>(i) * m, m, TM_MODE_KNN, k, merge_offset, 0.0f, 0u};
    tm_result *res = nullptr;
    const int rc = tm_scan_batch(ctx, reqs.data(), count, &res);
    if (rc != TM_OK)
        return rc;
    for (int i = 0; i < count; i++)
        for (int j = 0; j < k; j++)
        {
            const Hit h = res->answers[i].at(j);
            I[static_cast<size_t>(i) * k + j] = h.pos;
            D[static_cast<size_t>(i) * k + j] = h.dist;
        }
    tm_result_free(res);
    return TM_OK;
}

int tm_search_threshold(tm_ctx *ctx, const float *queries, int count, int m, float correlation, int merge_offset,
                        tm_result **out)
{
    if (ctx == nullptr || queries == nullptr || out == nullptr || count < 0)
        return TM_ERR_ARGUMENT;
    std::vector<tm_request> reqs(static_cast<size_t>(count));
    for (int i = 0; i < count; i++)
        reqs[i] = tm_request{queries + static_cast<size_t>(i) * m, m, TM_MODE_THRESHOLD, 1, merge_offset, correlation,
                             0u};
    return tm_scan_batch(ctx, reqs.data(), count, out);
}

int tm_result_count(const tm_result *res, int request, uint64_t *count)
{
    if (res == nullptr || count == nullptr || request < 0 || request >= static_cast<int>(res->answers.size()))
        return TM_ERR_ARGUMENT;
    *count = res->answers[request].size();
    return TM_OK;
}

int tm_result_get(const tm_result *res, int request, uint64_t *positions, float *distances, uint64_t capacity)
{
    if (res == nullptr || request < 0 || request >= static_cast<int>(res->answers.size()))
        return TM_ERR_ARGUMENT;
    const Answer &a = res->answers[request];
    if (capacity < a.size())
        return TM_ERR_CAPACITY;
    if (a.run)
    {
        if (positions)
            for (uint64_t i = 0; i < a.count; i++)
                positions[i] = a.w0 + a.win[i];
        if (distances && a.count > 0)
            std::memcpy(distances, a.dist, sizeof(float) * a.count);
        return TM_OK;
    }
    for (size_t i = 0; i < a.hits.size(); i++)
    {
        if (positions)
            positions[i] = a.hits[i].pos;
        if (distances)
            distances[i] = a.hits[i].dist;
    }
    return TM_OK;
}

void tm_result_free(tm_result *res) { delete res; }

float tm_cc_to_ed(float correlation, int m) { return tm_host::cc_to_ed(correlation, m); }
float tm_ed_to_cc(float distance, int m) { return tm_host::ed_to_cc(distance, m); }

int tm_profile_enable(tm_ctx *ctx, int enable)
{
    if (ctx == nullptr)
        return TM_ERR_ARGUMENT;
    ctx->main.profile = enable != 0;
    return TM_OK;
}

int tm_profile_read(tm_ctx *ctx, char *name, size_t name_capacity, int64_t *launches, double *milliseconds,
                    double *flops, int64_t *all_launches)
{
    if (ctx == nullptr)
        return TM_ERR_ARGUMENT;
    if (name && name_capacity > 0)
    {
        std::snprintf(name, name_capacity, "%s", ctx->main.kname.c_str());
    }
    if (launches)
        *launches = ctx->main.prof_launches;
    if (milliseconds)
        *milliseconds = ctx->main.prof_ms;
    if (flops)
        *flops = ctx->main.prof_flops;
    if (all_launches)
        *all_launches = ctx->main.all_launches;
    ctx->main.prof_launches = 0;
    ctx->main.prof_ms = 0.0;
    ctx->main.prof_flops = 0.0;
    ctx->main.all_launches = 0;
    return TM_OK;
}

int tm_profile_phases(tm_ctx *ctx, double *milliseconds, int capacity)
{
    if (ctx == nullptr || capacity < 0 || (capacity > 0 && milliseconds == nullptr))
        return TM_ERR_ARGUMENT;
    for (int i = 0; i < TM_PHASES; i++)
    {
        if (i < capacity)
            milliseconds[i] = ctx->main.phase_ms[i];
        ctx->main.phase_ms[i] = 0.0;
    }
    return TM_PHASES;
}

int tm_bound_diagnostics(tm_ctx *ctx, const float *queries, int count, int m, float *d, float *e, float *exact)
{
    if (ctx == nullptr || queries == nullptr || d == nullptr || e == nullptr || count < 1 || m < 1 ||
        static_cast<uint64_t>(m) > ctx->n)
        return TM_ERR_ARGUMENT;
    return guarded(ctx, [&] {
        TM_CUDA(cudaSetDevice(ctx->device));
        std::vector<tm_request> reqs(static_cast<size_t>(count));
        std::vector<int> idx(static_cast<size_t>(count));
        for (int i = 0; i < count; i++)
        {
            reqs[i] = tm_request{queries + static_cast<size_t>(i) * m, m, TM_MODE_THRESHOLD, 1, 0, 1.0f, 0u};
            idx[i] = i;
        }
        if (ctx->tiles >= TM_TILES_COLS_128 && ctx->kernel != TM_KERNEL_FP32 && tmb::umma_supported(m, count, 0) &&
            (ctx->tiles != TM_TILES_FFT || m <= tmb::kFftS))
        {
            bound_diagnostics_wm(ctx, m, idx, reqs, d, e, exact);
            return;
        }
        GroupPlan g;
        uint64_t h2d = 0;
        prepare_group(ctx, ctx->main, m, idx, reqs.data(), g, h2d);
        LengthStats &ls = ensure_length(ctx, ctx->main, m);
        const uint64_t W = ls.W;
        if (W == 0 || W * static_cast<uint64_t>(count) > (1ull << 31))
            throw Failure{TM_ERR_ARGUMENT, "diagnostics need 0 < windows x templates <= 2^31"};
        const bool use_umma = ctx->kernel != TM_KERNEL_FP32 && g.t_rows > 0 && tmb::umma_supported(m, count, W);
        for (int t = 0; t < count; t++)
        {
            g.htp[t].thr_ed = -FLT_MAX; // emit nothing
            if (use_umma)
                g.htp[t].a1_main = g.a1_umma[t];
        }
        cudaStream_t s = ctx->main.stream;
        TM_CUDA(cudaMemcpyAsync(g.tp.p, g.htp.data(), sizeof(TemplParam) * g.T_pad, cudaMemcpyHostToDevice, s));
        const size_t pairs = W * static_cast<size_t>(count);
        DevBuf dd, de, dc;
        dd.reserve(pairs * sizeof(float));
        de.reserve(pairs * sizeof(float));
        ctx->main.counters.reserve(4 * sizeof(uint32_t));
        TM_CUDA(cudaMemsetAsync(ctx->main.counters.p, 0, 4 * sizeof(uint32_t), s));
        TM_CUDA(cudaMemsetAsync(dd.p, 0xff, pairs * sizeof(float), s)); // NaN where nothing was written
        TM_CUDA(cudaMemsetAsync(de.p, 0xff, pairs * sizeof(float), s));
        ctx->main.cand.reserve(sizeof(Candidate) * 16);
        tmb::ScanArgs a{};
        a.x = ctx->clean.as<float>();
        a.q = g.q.as<float>();
        a.tp = g.tp.as<TemplParam>();
        a.mean = ls.mean.as<float>();
        a.inv = ls.inv.as<float>();
        a.w0 = ls.w0;
        a.W = static_cast<uint32_t>(W);
        a.m_pad = g.m_pad;
        a.T = count;
        a.nb = 1;
        a.cand = ctx->main.cand.as<Candidate>();
        a.cand_count = ctx->main.counters.as<uint32_t>();
        a.cand_cap = 0;
        a.q_hi = g.q_hi.p;
        a.q_lo = g.q_lo.p;
        a.t_rows = g.t_rows;
        a.err = reinterpret_cast<int *>(ctx->main.counters.as<uint32_t>() + 2);
        a.dbg_d = dd.as<float>();
        a.dbg_e = de.as<float>();
        TM_CUDA(use_umma ? tmb::launch_scan_umma(a, s) : tmb::launch_scan_fp32(a, s));
        count_launch(ctx->main);
        TM_CUDA(cudaMemcpyAsync(d, dd.p, pairs * sizeof(float), cudaMemcpyDeviceToHost, s));
        TM_CUDA(cudaMemcpyAsync(e, de.p, pairs * sizeof(float), cudaMemcpyDeviceToHost, s));
        if (exact != nullptr)
        {
            std::vector<Candidate> all(pairs);
            for (int t = 0; t < count; t++)
                for (uint64_t j = 0; j < W; j++)
                    all[static_cast<size_t>(t) * W + j] = Candidate{static_cast<uint32_t>(t), static_cast<uint32_t>(j)};
            dc.reserve(pairs * sizeof(Candidate));
            DevBuf dx;
            dx.reserve(pairs * sizeof(float));
            TM_CUDA(cudaMemcpyAsync(dc.p, all.data(), pairs * sizeof(Candidate), cudaMemcpyHostToDevice, s));
            TM_CUDA(tmb::launch_rescore(dc.as<Candidate>(), static_cast<uint32_t>(pairs), g.tp.as<TemplParam>(),
                                        g.q.as<float>(), g.order.as<int>(), ctx->raw.as<float>(), ls.w0, dx.as<float>(),
                                        s));
            count_launch(ctx->main);
            TM_CUDA(cudaMemcpyAsync(exact, dx.p, pairs * sizeof(float), cudaMemcpyDeviceToHost, s));
            TM_CUDA(cudaStreamSynchronize(s));
            dx.release();
        }
        uint32_t err = 0;
        TM_CUDA(cudaMemcpyAsync(&err, ctx->main.counters.as<uint32_t>() + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        TM_CUDA(cudaStreamSynchronize(s));
        dd.release();
        de.release();
        dc.release();
        g.release();
        if (err != 0)
            throw Failure{TM_ERR_TIMEOUT, "contraction kernel gave up waiting"};
    });
}

int tm_d2h_bytes(tm_ctx *ctx, uint64_t *bytes)
{
    if (ctx == nullptr || bytes == nullptr)
        return TM_ERR_ARGUMENT;
    *bytes = ctx->main.d2h_bytes;
    ctx->main.d2h_bytes = 0;
    return TM_OK;
}

int tm_ctx_stream(tm_ctx *ctx, void **stream)
{
    if (ctx == nullptr || stream == nullptr)
        return TM_ERR_ARGUMENT;
    *stream = static_cast<void *>(ctx->main.stream);
    return TM_OK;
}

int tm_last_candidates(const tm_ctx *ctx, uint64_t *count)
{
    if (ctx == nullptr || count == nullptr)
        return TM_ERR_ARGUMENT;
    *count = ctx->main.last_candidates;
    return TM_OK;
}


int tm_serve_start(tm_ctx *ctx, const tm_serve_config *config)
{
    if (ctx == nullptr)
        return TM_ERR_ARGUMENT;
    if (ctx->server && !ctx->server->stopped)
        return TM_ERR_STATE;
    tm_serve_config cfg{2, 256, 0};
    if (config)
        cfg = *config;
    if (cfg.workers < 1 || cfg.workers > 8 || cfg.max_batch < 1)
        return TM_ERR_ARGUMENT;
    return guarded(ctx, [&] {
        TM_CUDA(cudaSetDevice(ctx->device));
        if (ctx->kernel == TM_KERNEL_FP32 || !tmb::umma_supported(0, 0, 0))
            throw Failure{TM_ERR_STATE, "serving batches templates of several lengths on the tensor-core kernel"};
        ensure_prefix(ctx, ctx->main);
        if (cfg.memory_budget == 0)
        {
            size_t free_b = 0, total_b = 0;
            TM_CUDA(cudaMemGetInfo(&free_b, &total_b));
            cfg.memory_budget = free_b / 4;
        }
        ctx->server.reset();
        auto sv = std::make_unique<Server>();
        sv->ctx = ctx;
        sv->cfg = cfg;
        for (int i = 0; i < cfg.workers; i++)
        {
            sv->lanes.push_back(std::make_unique<Lane>());
            sv->lanes.back()->open();
        }
        Server *p = sv.get();
        ctx->server = std::move(sv);
        for (int i = 0; i < cfg.workers; i++)
            p->threads.emplace_back(serve_worker, p, p->lanes[i].get());
    });
}

int tm_submit(tm_ctx *ctx, const tm_request *request, uint64_t *ticket)
{
    if (ctx == nullptr || request == nullptr || ticket == nullptr)
        return TM_ERR_ARGUMENT;
    Server *sv = ctx->server.get();
    if (sv == nullptr || sv->stopped)
        return TM_ERR_STATE;
    const int rc = validate_requests(ctx, request, 1);
    if (rc != TM_OK)
        return rc;
    if (request->m > 16384)
        return TM_ERR_ARGUMENT;
    ServeItem it;
    try
    {
        it.templ.assign(request->templ, request->templ + request->m);
    }
    catch (const std::bad_alloc &)
    {
        return TM_ERR_NO_MEMORY;
    }
    it.req = *request;
    it.bytes = serve_bytes(ctx, *request);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stopping)
            return TM_ERR_STATE;
        it.ticket = sv->next_ticket++;
        it.submit_ms = sv->now_ms();
        *ticket = it.ticket;
        sv->pending.push_back(std::move(it));
    }
    sv->work_cv.notify_one();
    return TM_OK;
}

int tm_poll(tm_ctx *ctx, tm_completion *out, int capacity, int timeout_ms, int *count)
{
    if (ctx == nullptr || count == nullptr || capacity < 0 || (capacity > 0 && out == nullptr))
        return TM_ERR_ARGUMENT;
    *count = 0;
    Server *sv = ctx->server.get();
    if (sv == nullptr)
        return TM_ERR_STATE;
    std::unique_lock<std::mutex> lk(sv->mu);
    if (sv->done.empty() && timeout_ms != 0)
    {
        auto ready = [&] { return !sv->done.empty(); };
        if (timeout_ms < 0)
            sv->done_cv.wait(lk, ready);
        else
            sv->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    }
    int n = 0;
    while (n < capacity && !sv->done.empty())
    {
        out[n++] = sv->done.front();
        sv->done.pop_front();
    }
    *count = n;
    return TM_OK;
}

int tm_serve_stop(tm_ctx *ctx)
{
    if (ctx == nullptr)
        return TM_ERR_ARGUMENT;
    if (!ctx->server)
        return TM_ERR_STATE;
    stop_server(ctx);
    return TM_OK;
}

int tm_serve_status(tm_ctx *ctx, uint64_t *pending, uint64_t *in_flight, uint64_t *in_flight_bytes,
                    uint64_t *launches)
{
    if (ctx == nullptr)
        return TM_ERR_ARGUMENT;
    Server *sv = ctx->server.get();
    if (sv == nullptr)
        return TM_ERR_STATE;
    std::lock_guard<std::mutex> lk(sv->mu);
    if (pending)
        *pending = sv->pending.size();
    if (in_flight)
        *in_flight = sv->in_flight;
    if (in_flight_bytes)
        *in_flight_bytes = sv->in_flight_bytes;
    if (launches)
        *launches = sv->launches;
    return TM_OK;
}

} // extern "C"
