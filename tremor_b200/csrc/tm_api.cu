// C ABI of tremor_b200 (include/tremor_b200.h): context, window statistics, batched
// searches, results (serving: tm_serve.cu). One search of a group of same-length templates runs:
//
//   1. host: z-normalise each template (bit-identical to the reference), block order,
//      epilogue constants;                                        (tm_host.cpp)
//   2. device: contraction kernel with fused epilogue: threshold candidates and
//      per-bucket minima for kNN;                (tm_scan_fp32.cu / tm_scan_umma.cu)
//   3. device, kNN only: bound from bucket minima, list of buckets within it, FP32
//      re-pass of those buckets emitting the kNN candidates;        (tm_select.cu)
//   4. device: every candidate re-scored with the reference's exact arithmetic;
//   5. host: canonical exclusion selection / threshold merge on the exact distances.
#include "tm_core.h"

using namespace tmh;

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
        // per-batch buffers come from the context's own memory pool (DevBuf::reserve_on),
        // which keeps up to 4 GiB of freed memory for the next batch instead of returning
        // it to the driver at every synchronisation; the process's default pool is untouched
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        TM_CUDA(cudaMemPoolCreate(&ctx->pool, &props));
        uint64_t keep = 4ull << 30;
        TM_CUDA(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
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
                      &ctx->fft2_X, &ctx->fft2_shift, &ctx->fft2_norm, &ctx->fft3_X, &ctx->fft3_shift,
                      &ctx->fft3_norm, &ctx->fft_roots, &ctx->fft_scratch})
        b->release();
    // buffers of batches that outlive the context return to the pool when those batches
    // are destroyed; the driver releases the pool's memory once none is outstanding
    if (ctx->pool)
        cudaMemPoolDestroy(ctx->pool);
    delete ctx;
    return TM_OK;
}

const char *tm_last_error(const tm_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int tm_set_kernel(tm_ctx *ctx, int kernel)
{
    if (ctx == nullptr || kernel < TM_KERNEL_AUTO || kernel > TM_KERNEL_SPLIT_BF16)
        return TM_ERR_ARGUMENT;
    if (serving(ctx))
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
                    const int m = ks[ki] - (mixed ? t : 0); // several lengths: 128 distinct ones
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
        // the FFT branch, 8 templates of distinct lengths each (its time does not depend on
        // the length within either kind; distinct lengths share no window statistics, the
        // case of batches of many lengths): templates of up to 8192 samples (4089-4096 here)
        // and longer ones (16377-16384)
        tc->tiles = TM_TILES_FFT;
        double fft_per[2];
        for (int kind = 0; kind < 2; kind++)
        {
            std::vector<std::vector<float>> ft(8);
            std::vector<tm_request> fr(8);
            for (int t = 0; t < 8; t++)
            {
                const int m = (kind == 0 ? 4096 : 16384) - t;
                ft[t].resize(static_cast<size_t>(m));
                for (int i = 0; i < m; i++)
                    ft[t][i] = std::sin(0.003f * static_cast<float>(i) * (1.0f + 0.01f * t) +
                                        1e-6f * static_cast<float>(i) * static_cast<float>(i));
                fr[t] = tm_request{ft[t].data(), m, TM_MODE_THRESHOLD, 1, 0, 0.995f, 0u};
            }
            tm_batch b;
            create_batch(tc, tc->main, fr.data(), 8, b);
            tm_result res;
            run_batch(tc, tc->main, b, res);
            tc->main.profile = true;
            tc->main.prof_ms = 0.0;
            tc->main.prof_launches = 0;
            run_batch(tc, tc->main, b, res);
            tc->main.profile = false;
            fft_per[kind] = tc->main.prof_ms / 8.0 * (33554432.0 / static_cast<double>(n));
        }
        std::memcpy(ctx->tile_ms, table, sizeof(table));
        ctx->fft_ms = fft_per[0];
        ctx->fft_long_ms = fft_per[1];
        for (int i = 0; i < std::min(capacity, 34); i++)
            ms[i] = i < 32 ? (&table[0][0][0])[i] : fft_per[i - 32];
    });
    return rc == TM_OK ? 34 : rc;
}

int tm_set_tile_model(tm_ctx *ctx, const double *ms, int count)
{
    if (ctx == nullptr || ms == nullptr || count < 32 || count > 34)
        return TM_ERR_ARGUMENT;
    for (int i = 0; i < count; i++)
        if (!(ms[i] > 0.0) || !std::isfinite(ms[i]))
            return TM_ERR_ARGUMENT;
    std::memcpy(ctx->tile_ms, ms, sizeof(ctx->tile_ms));
    if (count >= 33)
        ctx->fft_ms = ms[32];
    if (count == 34)
        ctx->fft_long_ms = ms[33];
    return TM_OK;
}

int tm_set_window_range(tm_ctx *ctx, uint64_t first, uint64_t count)
{
    if (ctx == nullptr || count == 0)
        return TM_ERR_ARGUMENT;
    if (serving(ctx))
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

int tm_scan_knn(tm_ctx *ctx, const float *templ, int m, int k, int merge_offset, float bound_in, uint64_t *I,
                float *D)
{
    if (ctx == nullptr || templ == nullptr || I == nullptr || D == nullptr || k < 1 || std::isnan(bound_in))
        return TM_ERR_ARGUMENT;
    const int rc = tm_search_knn(ctx, templ, 1, m, k, merge_offset, I, D);
    if (rc != TM_OK)
        return rc;
    for (int j = 0; j < k; j++)
        if (!(D[j] <= bound_in))
        {
            I[j] = 0;
            D[j] = FLT_MAX;
        }
    return TM_OK;
}

int tm_scan_threshold(tm_ctx *ctx, const float *templ, int m, float correlation, int merge_offset, tm_result **out)
{
    return tm_search_threshold(ctx, templ, 1, m, correlation, merge_offset, out);
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
            (ctx->tiles != TM_TILES_FFT || m <= tmb::kFftMaxM))
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
        if (!use_umma)
        {
            ctx->main.fp32_qt.reserve(sizeof(float) * static_cast<size_t>(g.T_pad) * g.m_pad);
            a.qt = ctx->main.fp32_qt.as<float>();
            count_launch(ctx->main); // the template-tile transposition
        }
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


} // extern "C"
