/*
 * tremor_b200_worker_seam.hpp — the GPU branch of TREMOR's adaptive planner.
 *
 * The planner's worker (qa_exact_search_tremor_worker, tremor/algos/tremor/Tremor.cpp:2236-2318)
 * ends a template whose sampled candidate fraction calls for a scan in one of two branches,
 * refine_in_position_order (:1946, decision 1) or fft_in_position_order (:2088, decision 2);
 * both record the exact answers of the rank's owned windows in the worker's shared state.
 * tm_gpu_in_position_order is a drop-in for both calls: worker 0 searches the template over
 * the rank's windows on the GPU and records the answers where the CPU branches would, and
 * the other workers return at once to the barrier that follows (:2301).
 *
 *   threshold: every owned window with distance <= threshold_ed, unmerged, appended to
 *              threshold_hits under threshold_hits_lock (refine_in_position_order :2021-2026);
 *              the caller sorts and merges them by position as before (:2760-2795);
 *   kNN:       the template's canonical answers over the owned windows (k of them, the queue
 *              holding 2k - 1 with a merge offset, :2531), each offered through
 *              offer_knn_window (:1352-1362), so the candidate list and the bound queue hold
 *              them and the final select_knn_with_exclusion / rank gather (:341-408) run
 *              unchanged. Offering the exact top k of all windows to a candidate list that
 *              already holds other verified windows leaves the canonical selection unchanged:
 *              the greedy selection over any superset of its own answers returns them again.
 *
 * Which branch the planner would have taken (scan, with or without lower bounds, or FFT)
 * does not matter: the GPU chooses its own contraction (tensor-core tiles or the in-tree FFT
 * branch) from its measured model (tm_autotune), and every choice returns the same exact
 * answers. The windows the CPU scan skips (first sample missing, window past the chunk) are
 * the ones the library does not search either.
 *
 * Use: include this header inside Tremor.cpp after the definition of offer_knn_window (it
 * needs QaWorkerData and offer_knn_window), and call tm_gpu_in_position_order(in_data) at
 * both branch call sites. The rank's GPU context (its raw chunk, made resident once, with the
 * owned windows as its window range) is created on the first call and kept for the process;
 * TREMOR_GPU_DEVICE selects the device (default 0). A GPU failure ends the process with a
 * message, as the reference's CHECK_ALLOC does for allocation failures.
 */
#ifndef TREMOR_B200_WORKER_SEAM_HPP
#define TREMOR_B200_WORKER_SEAM_HPP

#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "tremor_b200.h"

namespace tm_seam
{
    struct State
    {
        std::mutex mu;
        tm_ctx *ctx = nullptr;
        const float *raw = nullptr; // the chunk the context holds
        idx_t chunk_length = 0, owned_first = 0, owned_count = 0;
    };

    inline State &state()
    {
        static State s;
        return s;
    }

    inline void fail(tm_ctx *ctx, int rc, const char *what)
    {
        std::fprintf(stderr, "tremor_b200: %s failed (%d): %s\n", what, rc, ctx ? tm_last_error(ctx) : "");
        std::exit(EXIT_FAILURE);
    }

    // The rank's context: its raw chunk resident on the GPU, searching the owned windows
    // (made again if the worker's chunk or owned range changes).
    inline tm_ctx *context(const QaWorkerData *in)
    {
        State &s = state();
        std::lock_guard<std::mutex> lk(s.mu);
        const idx_t first = in->local_owned_subseq_start - in->local_chunk_start;
        if (s.ctx != nullptr && s.raw == in->rawfile && s.chunk_length == in->local_chunk_length &&
            s.owned_first == first && s.owned_count == in->local_owned_subseq_count)
            return s.ctx;
        if (s.ctx != nullptr)
            tm_ctx_destroy(s.ctx);
        s.ctx = nullptr;
        const char *dev = std::getenv("TREMOR_GPU_DEVICE");
        int rc = tm_ctx_create(in->rawfile, static_cast<uint64_t>(in->local_chunk_length), dev ? std::atoi(dev) : 0,
                               &s.ctx);
        if (rc != TM_OK)
            fail(nullptr, rc, "tm_ctx_create");
        rc = tm_set_window_range(s.ctx, static_cast<uint64_t>(first), static_cast<uint64_t>(in->local_owned_subseq_count));
        if (rc != TM_OK)
            fail(s.ctx, rc, "tm_set_window_range");
        s.raw = in->rawfile;
        s.chunk_length = in->local_chunk_length;
        s.owned_first = first;
        s.owned_count = in->local_owned_subseq_count;
        return s.ctx;
    }
} // namespace tm_seam

// Drop-in for refine_in_position_order / fft_in_position_order (Tremor.cpp:1946, :2088).
static void tm_gpu_in_position_order(QaWorkerData *in)
{
    if (in->workernumber != 0)
        return;
    tm_ctx *ctx = tm_seam::context(in);
    const int m = in->index->settings->timeseries_size;
    pqueue_bsf *pq = in->bsf_result->pq_bsf;
    tm_request r{};
    r.templ = in->ts; // z-normalised by the caller (znormalize_inplace)
    r.m = m;
    r.flags = TM_FLAG_ZNORMALIZED;
    if (in->threshold_mode)
    {
        r.mode = TM_MODE_THRESHOLD;
        r.k = 1;
        r.merge_offset = 0; // every hit: the caller merges them as it merges the scan's
        r.correlation = in->corr_threshold;
    }
    else
    {
        r.mode = TM_MODE_KNN;
        r.merge_offset = in->merge_offset;
        r.k = in->merge_offset > 0 ? (pq->k + 1) / 2 : pq->k; // the queue holds 2k - 1 with a merge offset
    }
    tm_result *res = nullptr;
    int rc = tm_scan_batch(ctx, &r, 1, &res);
    if (rc != TM_OK)
        tm_seam::fail(ctx, rc, "tm_scan_batch");
    uint64_t n = 0;
    tm_result_count(res, 0, &n);
    std::vector<uint64_t> pos(n);
    std::vector<float> dist(n);
    rc = tm_result_get(res, 0, pos.data(), dist.data(), n);
    tm_result_free(res);
    if (rc != TM_OK)
        tm_seam::fail(ctx, rc, "tm_result_get");
    const file_position_type base = static_cast<file_position_type>(in->local_chunk_start); // chunk -> global
    std::printf("[Node %d] GPU branch: query %d, %llu %s\n", in->my_rank, in->query_counter,
                static_cast<unsigned long long>(n), in->threshold_mode ? "hits" : "answers");
    if (in->threshold_mode)
    {
        if (in->threshold_hits != nullptr && in->threshold_hits_lock != nullptr && n > 0)
        {
            pthread_mutex_lock(in->threshold_hits_lock);
            for (uint64_t i = 0; i < n; i++)
                in->threshold_hits->emplace_back(base + pos[i], dist[i]);
            pthread_mutex_unlock(in->threshold_hits_lock);
        }
        return;
    }
    // Answers of distance FLT_MAX are constant windows (the reference offers them while its
    // queue is not full), in position order, then (0, FLT_MAX) padding when the rank has fewer
    // than k windows; a (0, FLT_MAX) entry is a window only if window 0 is an owned, constant one.
    bool zero_seen = false;
    for (uint64_t i = 0; i < n; i++)
    {
        if (dist[i] == FLT_MAX && pos[i] == 0)
        {
            if (zero_seen)
                continue;
            zero_seen = true;
            const tm_seam::State &s = tm_seam::state();
            float mean = 0.0f, sd = 1.0f;
            if (s.owned_first != 0 || s.owned_count == 0 || in->rawfile[0] == TM_MISSING_VALUE ||
                tm_window_stats(ctx, m, 0, 1, &mean, &sd) != TM_OK || sd != 0.0f)
                continue;
        }
        offer_knn_window(in, pq, dist[i], base + pos[i], nullptr);
    }
}

#endif
