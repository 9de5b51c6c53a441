// Preparation of a batch's groups on the host: bit-identical template z-normalisation
// and block order (tm_host.cpp), the epilogue's error-bound constants, BF16 halves, row
// or column tiles of templates of several lengths, and the planner that splits each group
// between the FFT branch and a tile shape.
#include "tm_core.h"

namespace tmh {

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

// Host preparation of one group (bit-identical template z-normalisation and block
// order, epilogue constants) and its upload.
void prepare_group(tm_ctx *ctx, Lane &L, int m, const std::vector<int> &idx, const tm_request *reqs, GroupPlan &g,
                   uint64_t &h2d, int col_tile)
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
    g.q.reserve_on(sizeof(float) * static_cast<size_t>(T_pad) * m_pad, s, ctx->pool);
    g.order.reserve_on(sizeof(int) * static_cast<size_t>(T) * nblk, s, ctx->pool);
    g.tp.reserve_on(sizeof(TemplParam) * T_pad, s, ctx->pool);
    g.slots.reserve_on(sizeof(int) * std::max(g.nk, 1), s, ctx->pool);
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
        g.q_hi.reserve_on(sizeof(uint16_t) * elems, s, ctx->pool);
        g.q_lo.reserve_on(sizeof(uint16_t) * elems, s, ctx->pool);
        TM_CUDA(cudaMemcpyAsync(g.q_hi.p, hh, sizeof(uint16_t) * elems, cudaMemcpyHostToDevice, s));
        TM_CUDA(cudaMemcpyAsync(g.q_lo.p, hl, sizeof(uint16_t) * elems, cudaMemcpyHostToDevice, s));
        h2d += 2 * sizeof(uint16_t) * static_cast<uint64_t>(T) * m;
    }
    // the staging buffers are reused by the next group: finish the copies first
    TM_CUDA(cudaStreamSynchronize(s));
    h2d += sizeof(float) * static_cast<uint64_t>(T) * m + sizeof(int) * static_cast<uint64_t>(T) * nblk +
           sizeof(TemplParam) * T_pad;
}

// Host preparation of a mixed-length group: templates sorted by length (longest first),
// in tiles of 128 rows (col_tile 0, k_scan_umma) or col_tile rows (k_scan_wm), any
// lengths. Padding rows are inert; a tile's K extent is its longest template (shorter rows are
// zero-padded, which leaves their dot products unchanged). Rows are the template slots of
// the group: g.index[row] is the request (-1 for padding rows).
void prepare_group_mixed(tm_ctx *ctx, Lane &L, const std::vector<int> &idx_in, const tm_request *reqs, GroupPlan &g,
                         uint64_t &h2d, int col_tile)
{
    std::vector<int> idx = idx_in;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return reqs[a].m > reqs[b].m; });
    const size_t tile_rows = col_tile > 0 ? static_cast<size_t>(col_tile) : 128;
    // rows: request per row (-1 = padding)
    std::vector<int> rows;
    std::vector<tmb::TileInfo> tiles;
    std::vector<int> tile_len; // the longest template of each tile
    for (size_t i = 0; i < idx.size();)
    {
        const size_t start = rows.size();
        const int longest = reqs[idx[i]].m;
        while (i < idx.size() && rows.size() - start < tile_rows)
            rows.push_back(idx[i++]);
        while (rows.size() - start < tile_rows)
            rows.push_back(-1);
        tiles.push_back(tmb::TileInfo{(longest + 63) / 64});
        tile_len.push_back(longest);
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
        if (rows[t] < 0)
        {
            p.mode = TM_MODE_THRESHOLD;
            p.thr_ed = -FLT_MAX;
            p.m = tile_len[static_cast<size_t>(t) / tile_rows];
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
    g.tiles = tiles;
    cudaStream_t s = L.stream;
    g.q.reserve_on(sizeof(float) * elems, s, ctx->pool);
    g.order.reserve_on(sizeof(int) * static_cast<size_t>(R) * nblk, s, ctx->pool);
    g.tp.reserve_on(sizeof(TemplParam) * R, s, ctx->pool);
    g.slots.reserve_on(sizeof(int) * std::max(g.nk, 1), s, ctx->pool);
    g.q_hi.reserve_on(sizeof(uint16_t) * elems, s, ctx->pool);
    g.q_lo.reserve_on(sizeof(uint16_t) * elems, s, ctx->pool);
    g.d_tiles.reserve_on(sizeof(tmb::TileInfo) * tiles.size(), s, ctx->pool);
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
int plan_col_tile(const tm_ctx *ctx, const tm_request *reqs, const std::vector<int> &idx, double *cost)
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
        if (reqs[i].m > tmb::kFftMaxM)
            return 0;
    if (ctx->tiles == TM_TILES_FFT)
        return n;
    if (ctx->tiles != TM_TILES_AUTO || ctx->kernel != TM_KERNEL_AUTO)
        return 0;
    std::vector<int> m(n);
    for (size_t i = 0; i < n; i++)
        m[i] = reqs[sorted_idx[i]].m;
    size_t best_f = 0;
    double best = tensor_cost_sorted(ctx, m.data(), n), fft_cost = 0.0;
    for (size_t f = 1; f <= n; f++)
    {
        // the fused kernels take templates of up to 8192 samples; longer ones cost more
        fft_cost += m[f - 1] <= tmb::kF2S ? ctx->fft_ms : ctx->fft_long_ms;
        const double c = fft_cost + tensor_cost_sorted(ctx, m.data() + f, n - f);
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
void create_batch(tm_ctx *ctx, Lane &L, const tm_request *requests, int count, tm_batch &b, bool serving)
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
    for (size_t gi = specs.size(); gi < b.groups.size(); gi++) // a reused batch with fewer groups
        b.groups[gi].release();
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

} // namespace tmh
