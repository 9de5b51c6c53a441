// The device pipeline of a prepared group: window statistics (per length, or the
// resident prefix sums), the contraction kernel or the FFT branch with its bounded
// epilogue, the kNN bound and FP32 re-pass, exact re-scoring, and the answers assembled on
// the device and handed to the result in pinned memory.
#include <unordered_map>
#include "tm_core.h"

namespace tmh {

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
        {
            L.fp32_qt.reserve(sizeof(float) * static_cast<size_t>(g.T_pad) * g.m_pad);
            a.qt = L.fp32_qt.as<float>();
            TM_CUDA(tmb::launch_scan_fp32(a, s));
            count_launch(L); // the template-tile transposition
        }
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

// Spectra of the record's pieces for the FFT branch (tm_fftk.cu), their shifts and norms,
// and the twiddle tables: built once per context and piece length (long = pieces of 32768
// samples every 16384, else 16384 every 8192), under a lock (serving workers may ask at once).
static void ensure_fft(tm_ctx *ctx, Lane &L, bool long_pieces)
{
    std::lock_guard<std::mutex> lk(ctx->fft_mu);
    if (long_pieces ? ctx->fft3_ready : ctx->fft2_ready)
        return;
    ensure_prefix(ctx, L);
    cudaStream_t s = L.stream;
    if (ctx->fft_roots.p == nullptr)
    {
        std::vector<double2> roots(tmb::kFftRoots);
        tmb::fft_roots(roots.data());
        ctx->fft_roots.reserve(sizeof(double2) * tmb::kFftRoots);
        TM_CUDA(cudaMemcpyAsync(ctx->fft_roots.p, roots.data(), sizeof(double2) * tmb::kFftRoots,
                                cudaMemcpyHostToDevice, s));
        int sms = 0;
        TM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        ctx->sms = sms;
        ctx->fft_scratch.reserve(sizeof(double2) * static_cast<size_t>(sms) * tmb::kFftScratchPts);
    }
    const uint32_t B = 16384; // pieces per launch
    if (!long_pieces)
    {
        const uint32_t P = tmb::fft2_pieces(ctx->n);
        ctx->fft2_X.reserve(sizeof(double2) * static_cast<size_t>(P) * tmb::kF2H);
        ctx->fft2_shift.reserve(sizeof(double) * P);
        ctx->fft2_norm.reserve(sizeof(double) * P);
        for (uint32_t p0 = 0; p0 < P; p0 += B)
        {
            TM_CUDA(tmb::launch_fft2_pieces(ctx->clean.as<float>(), ctx->n, ctx->pcen.as<double>(), p0,
                                            std::min<uint32_t>(B, P - p0), ctx->fft_roots.as<double2>(),
                                            ctx->fft2_X.as<double2>(), ctx->fft2_shift.as<double>(),
                                            ctx->fft2_norm.as<double>(), s));
            count_launch(L);
        }
        ctx->fft2_P = P;
    }
    else
    {
        const uint32_t P = tmb::fft3_pieces(ctx->n);
        ctx->fft3_X.reserve(sizeof(double2) * static_cast<size_t>(P) * tmb::kF3H);
        ctx->fft3_shift.reserve(sizeof(double) * P);
        ctx->fft3_norm.reserve(sizeof(double) * P);
        for (uint32_t p0 = 0; p0 < P; p0 += B)
        {
            TM_CUDA(tmb::launch_fft3_pieces(ctx->clean.as<float>(), ctx->n, ctx->pcen.as<double>(), p0,
                                            std::min<uint32_t>(B, P - p0), ctx->fft_roots.as<double2>(),
                                            ctx->fft3_X.as<double2>(), ctx->fft3_shift.as<double>(),
                                            ctx->fft3_norm.as<double>(), ctx->fft_scratch.as<double2>(), ctx->sms,
                                            s));
            count_launch(L);
        }
        ctx->fft3_P = P;
    }
    TM_CUDA(cudaStreamSynchronize(s));
    (long_pieces ? ctx->fft3_ready : ctx->fft2_ready) = true;
}

// The FFT branch for the group's rows `rows` (all of up to 8192 samples, or all longer):
// their spectra, then one persistent launch over the pieces their windows touch.
static void fft_contract_rows(tm_ctx *ctx, Lane &L, const GroupPlan &g, const tmb::ScanArgs &a,
                              const std::vector<int> &rows, bool long_pieces)
{
    ensure_fft(ctx, L, long_pieces);
    cudaStream_t s = L.stream;
    const int nr = static_cast<int>(rows.size());
    const size_t H = long_pieces ? tmb::kF3H : tmb::kF2H;
    const uint32_t S = long_pieces ? tmb::kF3S : tmb::kF2S;
    DevBuf &Y = long_pieces ? L.fft3_Y : L.fft2_Y;
    Y.reserve(sizeof(double2) * static_cast<size_t>(nr) * H);
    L.fft_rows.reserve(sizeof(int) * static_cast<size_t>(nr));
    L.fft_stats.reserve(sizeof(float4) * static_cast<size_t>(ctx->sms) * tmb::kFftCache);
    TM_CUDA(cudaMemcpyAsync(L.fft_rows.p, rows.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, s));
    // per row, the largest bound coefficients of the rows of its length (the epilogue's
    // folded window statistics serve every template of one length in a piece)
    std::vector<float4> gmax(2 * static_cast<size_t>(g.T), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    std::unordered_map<int, std::pair<float4, float4>> by_m;
    for (int t : rows)
    {
        const TemplParam &q = g.htp[static_cast<size_t>(t)];
        auto it = by_m.emplace(q.m, std::make_pair(make_float4(0.0f, 0.0f, 0.0f, 0.0f),
                                                   make_float4(0.0f, 0.0f, 0.0f, 0.0f))).first;
        float4 &c0 = it->second.first, &c1 = it->second.second;
        c0 = make_float4(std::max(c0.x, q.a1_main), std::max(c0.y, q.a2), std::max(c0.z, q.a5), std::max(c0.w, q.a6));
        c1 = make_float4(std::max(c1.x, q.qs), std::max(c1.y, std::fabs(q.s1)), 0.0f, 0.0f);
    }
    for (int t : rows)
    {
        const auto &c = by_m.at(g.htp[static_cast<size_t>(t)].m);
        gmax[2 * static_cast<size_t>(t)] = c.first;
        gmax[2 * static_cast<size_t>(t) + 1] = c.second;
    }
    L.fft_gmax.reserve(sizeof(float4) * gmax.size());
    TM_CUDA(cudaMemcpyAsync(L.fft_gmax.p, gmax.data(), sizeof(float4) * gmax.size(), cudaMemcpyHostToDevice, s));
    if (long_pieces)
    {
        // the forward transform's scratch is the context's: one launch at a time
        std::lock_guard<std::mutex> lk(ctx->fft_mu);
        TM_CUDA(tmb::launch_fft3_templates(g.q.as<float>(), g.tp.as<TemplParam>(), L.fft_rows.as<int>(), nr,
                                           ctx->fft_roots.as<double2>(), Y.as<double2>(),
                                           ctx->fft_scratch.as<double2>(), ctx->sms, s));
        TM_CUDA(cudaStreamSynchronize(s));
    }
    else
        TM_CUDA(tmb::launch_fft2_templates(g.q.as<float>(), g.tp.as<TemplParam>(), L.fft_rows.as<int>(), nr,
                                           ctx->fft_roots.as<double2>(), Y.as<double2>(), s));
    uint64_t wmax = 0;
    for (int t : rows)
        wmax = std::max<uint64_t>(wmax, g.htp[static_cast<size_t>(t)].wcount);
    const uint32_t P = long_pieces ? ctx->fft3_P : ctx->fft2_P;
    const uint64_t first = a.w0, last = a.w0 + wmax - 1;
    const uint32_t pa = static_cast<uint32_t>(first / S);
    const uint32_t pb = std::min<uint32_t>(static_cast<uint32_t>(last / S), P - 1);
    tmb::Fft2Args f{};
    f.X = (long_pieces ? ctx->fft3_X : ctx->fft2_X).as<double2>();
    f.shifts = (long_pieces ? ctx->fft3_shift : ctx->fft2_shift).as<double>();
    f.norms = (long_pieces ? ctx->fft3_norm : ctx->fft2_norm).as<double>();
    f.p_first = pa;
    f.p_count = pb >= pa ? pb - pa + 1 : 0;
    f.Y = Y.as<double2>();
    f.rows = L.fft_rows.as<int>();
    f.nrows = nr;
    f.tp = g.tp.as<TemplParam>();
    f.roots = ctx->fft_roots.as<double2>();
    f.w0 = a.w0;
    f.W = a.W;
    f.pv = tmb::PrefixView{a.P, a.PT, a.PC};
    f.run = a.run;
    f.raw = a.raw;
    f.bmin_u = a.bmin_u;
    f.bmin_l = a.bmin_l;
    f.nb = a.nb;
    f.cand = a.cand;
    f.cand_count = a.cand_count;
    f.cand_cap = a.cand_cap;
    f.dbg_d = a.dbg_d;
    f.dbg_e = a.dbg_e;
    f.stats = L.fft_stats.as<float4>();
    f.gmax = L.fft_gmax.as<float4>();
    TM_CUDA(long_pieces ? tmb::launch_fft3_corr(f, ctx->sms, s) : tmb::launch_fft2_corr(f, ctx->sms, s));
    count_launch(L, 2);
}

void fft_contract(tm_ctx *ctx, Lane &L, const GroupPlan &g, const tmb::ScanArgs &a)
{
    // templates of up to 8192 samples: pieces of 16384 samples; longer ones: pieces of 32768
    std::vector<int> short_rows, long_rows;
    for (int t = 0; t < g.T; t++)
    {
        const TemplParam &p = g.htp[t];
        if (g.index[t] < 0 || p.wcount == 0)
            continue;
        (p.m <= tmb::kF2S ? short_rows : long_rows).push_back(t);
    }
    if (!short_rows.empty())
        fft_contract_rows(ctx, L, g, a, short_rows, false);
    if (!long_rows.empty())
        fft_contract_rows(ctx, L, g, a, long_rows, true);
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

} // namespace tmh
