// Host-side internals of libtremor_b200 shared by its translation units: device and
// pinned buffers, results, lanes (a search in flight), the context, prepared groups and
// batches, and the functions one file calls in another.
//   tm_groups.cu  template preparation (bit-identical z-normalisation, block order,
//                 epilogue constants), tile-shape and FFT planning, batch creation
//   tm_search.cu  window statistics, the device pipeline of a group (contraction or FFT
//                 branch, kNN bound and re-pass, exact re-scoring, answer assembly)
//   tm_serve.cu   continuous batching (tm_serve_*)
//   tm_api.cu     the rest of the C ABI
#pragma once

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

namespace tmh {

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
    bool pooled = false; // from the device's memory pool (reserve_on)
    void reserve(size_t need)
    {
        if (need <= bytes)
            return;
        release();
        size_t b = std::max<size_t>(need, 256);
        TM_CUDA(cudaMalloc(&p, b));
        bytes = b;
    }
    // Stream-ordered allocation from a memory pool (the context's own), for the buffers
    // of one batch: freeing returns the memory to the pool without the device-wide
    // synchronisation and unmapping of cudaFree (tens of milliseconds with a large
    // context), and the next batch's allocation takes it back from there. A buffer that
    // grows is freed after the work already queued on s.
    void reserve_on(size_t need, cudaStream_t s, cudaMemPool_t pool)
    {
        if (need <= bytes)
            return;
        drop(s);
        size_t b = std::max<size_t>(need, 256);
        TM_CUDA(cudaMallocFromPoolAsync(&p, b, pool, s));
        bytes = b;
        pooled = true;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
    // Callers release only after the work that used the buffer has completed.
    void release() { drop(0); }
    // Stream-ordered release of a pooled buffer: after the work already queued on s.
    void release_on(cudaStream_t s) { drop(s); }

  private:
    void drop(cudaStream_t s)
    {
        if (p)
        {
            if (pooled)
                cudaFreeAsync(p, s);
            else
                cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
        pooled = false;
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

} // namespace tmh

namespace tmh {

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

} // namespace tmh

struct tm_result
{
    std::vector<tmh::Answer> answers;
    std::vector<std::shared_ptr<tmh::PinnedBlock>> blocks;
};

namespace tmh {

// The device state of one search in flight: a stream, its events, the search's scratch
// buffers and pinned staging, and its counters. The synchronous calls use the context's
// main lane; each serving worker owns one more, so searches on different lanes overlap
// (one's host work and copies with another's kernels).
struct Lane
{
    cudaStream_t stream = nullptr;
    DevBuf tkey, bmin_u, bmin_l, list, counters, cand, dist, fp32_qt; // (fp32_qt: k_scan_fp32's template tiles)
    // answer assembly: sort keys and values (double buffers), sort scratch, runs
    DevBuf akeys, avals, avals64, sort_tmp, segs;
    std::vector<std::shared_ptr<PinnedBlock>> pool;
    HostBuf h_split, h_q, h_order, h_slots, h_counters;
    uint32_t cand_cap = 1u << 22, list_cap = 1u << 20;
    // FFT branch: the template spectra and rows of a launch (both piece lengths)
    DevBuf fft2_Y, fft3_Y, fft_rows, fft_stats, fft_gmax; // (fft_stats: the correlation kernels' per-block statistics cache; fft_gmax: per row, its length's largest bound coefficients)
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
        for (DevBuf *b : {&tkey, &bmin_u, &bmin_l, &list, &counters, &cand, &dist, &fp32_qt, &akeys, &avals, &avals64, &sort_tmp,
                          &segs, &fft2_Y, &fft3_Y, &fft_rows, &fft_stats, &fft_gmax})
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

} // namespace tmh

struct tm_ctx
{
    int device = 0;
    uint64_t n = 0;
    tmh::DevBuf raw, clean;
    uint64_t range_first = 0, range_count = UINT64_MAX;
    int kernel = TM_KERNEL_AUTO;
    int tiles = TM_TILES_AUTO;
    // tiling cost model: kernel milliseconds for 128 templates x 2^25 windows, per group kind
    // (one length / several: 128 distinct lengths), shape (row tiles; column tiles of 128, 64,
    // 32) and K (256, 1024, 4096, 16384). Defaults: a B200 measurement; tm_autotune
    // re-measures.
    double tile_ms[2][4][4] = {{{7.2, 16.4, 58.7, 259.0},
                                {29.7, 31.5, 84.2, 334.1},
                                {31.5, 42.8, 157.6, 588.2},
                                {36.0, 83.2, 307.2, 1142.8}},
                               {{47.4, 53.6, 85.9, 274.6},
                                {70.8, 73.6, 89.2, 342.9},
                                {72.7, 75.1, 155.0, 583.7},
                                {78.3, 87.6, 310.9, 1163.1}}};
    std::map<int, std::unique_ptr<tmh::LengthStats>> lengths;
    uint64_t use_clock = 0;
    tmh::DevBuf suf; // window-statistics scratch (per-length statistics)
    // length-independent statistics (mixed-length batches): block-local FP64 prefix sums,
    // their block totals and centres, constant runs
    tmh::DevBuf prefix, ptot, pcen, run;
    bool prefix_ready = false;
    // FFT branch (tm_fftk.cu), built on first use: spectra of pieces of 16384 samples every
    // 8192 (templates of up to 8192 samples) and of pieces of 32768 every 16384 (longer ones),
    // their shifts and norms; the twiddle tables; the forward transforms' scratch
    tmh::DevBuf fft2_X, fft2_shift, fft2_norm, fft3_X, fft3_shift, fft3_norm, fft_roots, fft_scratch;
    uint32_t fft2_P = 0, fft3_P = 0;
    bool fft2_ready = false, fft3_ready = false;
    std::mutex fft_mu;
    int sms = 148;
    // model: the FFT branch's ms per template per 2^25 samples, for templates of up to 8192
    // samples (the fused kernels) and longer ones, templates of distinct lengths (B200 defaults;
    // tm_autotune measures both)
    double fft_ms = 0.71;
    double fft_long_ms = 1.07;
    // the context's own memory pool for per-batch buffers (DevBuf::reserve_on); it keeps
    // up to 4 GiB of freed memory for the next batch
    cudaMemPool_t pool = nullptr;
    std::string err;
    tmh::Lane main;                      // the synchronous calls' lane
    // serving engine, while started; replaced only under server_mu, and the serving calls
    // take their own reference under it, so a restart cannot free a server in use
    std::shared_ptr<tmh::Server> server;
    std::mutex server_mu;

    tm_ctx();  // both in tm_serve.cu, where the server's type is complete
    ~tm_ctx();
};

namespace tmh {

inline int fail(tm_ctx *ctx, const Failure &f)
{
    if (ctx)
        ctx->err = f.what;
    return f.code;
}

template <class F> inline int guarded(tm_ctx *ctx, F body)
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

inline void count_launch(Lane &L, int k = 1) { L.all_launches += k; }

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
    std::vector<tmb::TileInfo> tiles; // per tile: K blocks
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

} // namespace tmh

struct tm_batch
{
    int count = 0;
    std::vector<tmh::GroupPlan> groups;
    uint64_t h2d_bytes = 0;
    ~tm_batch()
    {
        for (tmh::GroupPlan &g : groups)
            g.release();
    }
};

namespace tmh {

// tm_search.cu
LengthStats &ensure_length(tm_ctx *ctx, Lane &L, int m);
void ensure_prefix(tm_ctx *ctx, Lane &L);
void fft_contract(tm_ctx *ctx, Lane &L, const GroupPlan &g, const tmb::ScanArgs &a);
void run_batch(tm_ctx *ctx, Lane &L, tm_batch &b, tm_result &res);
int validate_requests(const tm_ctx *ctx, const tm_request *reqs, int count);

// tm_groups.cu
void prepare_group(tm_ctx *ctx, Lane &L, int m, const std::vector<int> &idx, const tm_request *reqs, GroupPlan &g,
                   uint64_t &h2d, int col_tile = 0);
void prepare_group_mixed(tm_ctx *ctx, Lane &L, const std::vector<int> &idx_in, const tm_request *reqs, GroupPlan &g,
                         uint64_t &h2d, int col_tile = 0);
int plan_col_tile(const tm_ctx *ctx, const tm_request *reqs, const std::vector<int> &idx, double *cost = nullptr);
double tile_time(const tm_ctx *ctx, bool mixed, int v, double k);
void create_batch(tm_ctx *ctx, Lane &L, const tm_request *requests, int count, tm_batch &b, bool serving = false);

// tm_serve.cu
void stop_server(tm_ctx *ctx);
bool serving(tm_ctx *ctx);

} // namespace tmh
