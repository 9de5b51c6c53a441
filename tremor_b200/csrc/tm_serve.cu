#include "tm_core.h"

tm_ctx::tm_ctx() = default;
tm_ctx::~tm_ctx() = default;

namespace tmh {
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
    uint64_t bytes = 0;   // admission estimate of its device memory
    double cost_ms = 0.0; // and of its device time (serve_cost)
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

// Modelled device milliseconds of a request: the cheaper of the FFT branch (a constant per
// template, by kind) and its share of a full 128-row tile of mixed lengths at its own K, from
// the planner's model (ms per 2^25 windows), scaled to the record's windows.
static double serve_cost(const tm_ctx *ctx, const tm_request &r)
{
    const double scale = static_cast<double>(ctx->n - static_cast<uint64_t>(r.m) + 1) / 33554432.0;
    const double fft = r.m <= tmb::kF2S ? ctx->fft_ms : ctx->fft_long_ms;
    const double row = tile_time(ctx, true, 0, static_cast<double>((r.m + 63) & ~63)) / 128.0;
    return std::min(fft, row) * scale;
}

// Admission (under the server's lock). A batch is built a tile at a time: the 128 rows of
// a contraction tile share one K extent, their longest template, so rows not longer than
// that cost nothing extra. Each tile opens with the oldest pending request (so every batch
// admits the oldest, and later arrivals never hold a request back indefinitely) and fills
// with the longest pending requests not longer than it; with a long queue the tiles hold
// similar lengths.
// Stops at max_batch, at the memory budget or at the batch's modelled time (batch_ms); a
// first request alone is always admitted.
static void admit(Server *sv, std::vector<ServeItem> &batch, uint64_t &bytes)
{
    double ms = 0.0;
    for (const ServeItem &it : batch)
        ms += it.cost_ms;
    auto fits = [&](const ServeItem &it) {
        if (batch.empty() && sv->in_flight_bytes == 0)
            return true;
        if (sv->cfg.batch_ms > 0.0 && !batch.empty() && ms + it.cost_ms > sv->cfg.batch_ms)
            return false;
        return sv->in_flight_bytes + bytes + it.bytes <= sv->cfg.memory_budget;
    };
    std::vector<size_t> order;
    std::vector<char> chosen;
    while (!sv->pending.empty() && static_cast<int>(batch.size()) < sv->cfg.max_batch)
    {
        if (!fits(sv->pending.front()))
            return;
        const int cap_m = sv->pending.front().req.m;
        bytes += sv->pending.front().bytes;
        ms += sv->pending.front().cost_ms;
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
            if (taken == room || !fits(sv->pending[i]))
                break;
            bytes += sv->pending[i].bytes;
            ms += sv->pending[i].cost_ms;
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

// The context's current server (or null), by a reference taken under the context's lock.
static std::shared_ptr<Server> current_server(tm_ctx *ctx)
{
    std::lock_guard<std::mutex> lk(ctx->server_mu);
    return ctx->server;
}

// Completes what was submitted, then joins the workers; completions stay pollable, and a
// consumer waiting in tm_poll without a limit is woken once nothing is left to complete.
void stop_server(tm_ctx *ctx)
{
    std::shared_ptr<Server> sv = current_server(ctx);
    if (!sv)
        return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stopping)
            return; // stopped, or being stopped by another thread
        sv->stopping = true;
    }
    sv->work_cv.notify_all();
    for (std::thread &t : sv->threads)
        t.join();
    sv->threads.clear();
    for (auto &L : sv->lanes)
        L->close();
    sv->lanes.clear();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stopped = true;
    }
    sv->done_cv.notify_all();
}


bool serving(tm_ctx *ctx)
{
    std::shared_ptr<Server> sv = current_server(ctx);
    if (!sv)
        return false;
    std::lock_guard<std::mutex> lk(sv->mu);
    return !sv->stopped;
}

} // namespace tmh

using namespace tmh;

extern "C" {

int tm_serve_start(tm_ctx *ctx, const tm_serve_config *config)
{
    if (ctx == nullptr)
        return TM_ERR_ARGUMENT;
    if (serving(ctx))
        return TM_ERR_STATE;
    tm_serve_config cfg{1, 256, 0, 0.0};
    if (config)
        cfg = *config;
    if (cfg.workers < 1 || cfg.workers > 8 || cfg.max_batch < 1 || !(cfg.batch_ms >= 0.0))
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
        auto sv = std::make_shared<Server>();
        sv->ctx = ctx;
        sv->cfg = cfg;
        for (int i = 0; i < cfg.workers; i++)
        {
            sv->lanes.push_back(std::make_unique<Lane>());
            sv->lanes.back()->open();
        }
        Server *p = sv.get();
        {
            // the previous (stopped) server is freed once no serving call holds it
            std::lock_guard<std::mutex> lk(ctx->server_mu);
            ctx->server = std::move(sv);
        }
        for (int i = 0; i < cfg.workers; i++)
            p->threads.emplace_back(serve_worker, p, p->lanes[i].get());
    });
}

int tm_submit(tm_ctx *ctx, const tm_request *request, uint64_t *ticket)
{
    if (ctx == nullptr || request == nullptr || ticket == nullptr)
        return TM_ERR_ARGUMENT;
    std::shared_ptr<Server> sv = current_server(ctx);
    if (!sv)
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
    it.cost_ms = serve_cost(ctx, *request);
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
    std::shared_ptr<Server> sv = current_server(ctx);
    if (!sv)
        return TM_ERR_STATE;
    std::unique_lock<std::mutex> lk(sv->mu);
    if (sv->done.empty() && timeout_ms != 0)
    {
        // a stopped server completes nothing more: return instead of waiting for good
        auto ready = [&] { return !sv->done.empty() || sv->stopped; };
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
    if (!current_server(ctx))
        return TM_ERR_STATE;
    stop_server(ctx);
    return TM_OK;
}

int tm_serve_status(tm_ctx *ctx, uint64_t *pending, uint64_t *in_flight, uint64_t *in_flight_bytes,
                    uint64_t *launches)
{
    if (ctx == nullptr)
        return TM_ERR_ARGUMENT;
    std::shared_ptr<Server> sv = current_server(ctx);
    if (!sv)
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
