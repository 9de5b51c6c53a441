// C entry points around the reference's OWN scan code, compiled from the
// reference sources where they lie (see oracle/Makefile, target `ref`).
// Oracle infrastructure only: the tests and the CPU-baseline leg of bench.py
// load the resulting oracle/_ref/libtremor_ref.so; the product never does.
//
//   tmref_sss_knn / tmref_sss_threshold : SkipSequentialScan (SkipSequential.hpp:32-78)
//       built from a waveform file, one object per call (the template counter is
//       not reset between searches, SkipSequential.cpp:127-136).
//   tmref_sss_stats                      : the per-window statistics that
//       SkipSequentialScan::build computes (SkipSequential.cpp:157-190).
//   tmref_sss_from_stats / tmref_sss_distances : the same class over a record in memory
//       with given statistics (records too large for build()'s statistics in a test), and
//       the reference's distance at given windows.
//   tmref_l2_dist / tmref_znormalize / tmref_block_order / tmref_select_knn :
//       the inline building blocks of ZnormSearch.hpp, for bit-level pinning.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#define private public // read the statistics SkipSequentialScan::build keeps
#include "tremor/algos/sss/SkipSequential.hpp"
#undef private
#include "tremor/distance_computers/ZnormSearch.hpp"
#include "tremor/isax/iSAXPqueue.hpp"

extern "C"
{
    int tmref_sss_knn(const char *waveform_file, uint64_t total_samples, int m, const float *queries, int query_count,
                      int k, int merge_offset, int lower_bounds, int threads, int paa_segments, const char *out_csv)
    {
        try
        {
            SkipSequentialScan scan(threads, paa_segments, merge_offset, 0, lower_bounds != 0);
            scan.build(waveform_file, total_samples, m);
            scan.search_knn(queries, query_count, k, out_csv);
            return 0;
        }
        catch (const std::exception &)
        {
            return -1;
        }
    }

    int tmref_sss_threshold(const char *waveform_file, uint64_t total_samples, int m, const float *queries,
                            int query_count, float correlation, int merge_offset, int lower_bounds, int threads,
                            int paa_segments, const char *out_prefix)
    {
        try
        {
            SkipSequentialScan scan(threads, paa_segments, merge_offset, 0, lower_bounds != 0);
            scan.build(waveform_file, total_samples, m);
            scan.search_threshold(queries, query_count, correlation, out_prefix);
            return 0;
        }
        catch (const std::exception &)
        {
            return -1;
        }
    }

    int tmref_sss_stats(const char *waveform_file, uint64_t total_samples, int m, int threads, float *means,
                        float *stds)
    {
        try
        {
            SkipSequentialScan scan(threads, 8, 0, 0, false);
            scan.build(waveform_file, total_samples, m);
            std::memcpy(means, scan.means.data(), scan.means.size() * sizeof(float));
            std::memcpy(stds, scan.stds.data(), scan.stds.size() * sizeof(float));
            return 0;
        }
        catch (const std::exception &)
        {
            return -1;
        }
    }

    // A scan built once (SkipSequentialScan::build) and searched many times, with the
    // template counter rewound between searches; the searches are timed alone.
    void *tmref_sss_create(const char *waveform_file, uint64_t total_samples, int m, int k_unused, int merge_offset,
                           int lower_bounds, int threads, int paa_segments)
    {
        (void)k_unused;
        try
        {
            auto *scan = new SkipSequentialScan(threads, paa_segments, merge_offset, 0, lower_bounds != 0);
            scan->build(waveform_file, total_samples, m);
            return scan;
        }
        catch (const std::exception &)
        {
            return nullptr;
        }
    }

    // Seconds of SkipSequentialScan::search_knn / search_threshold (negative on failure).
    double tmref_sss_search(void *handle, const float *queries, int query_count, int knn, int k, float correlation,
                            const char *out)
    {
        auto *scan = static_cast<SkipSequentialScan *>(handle);
        try
        {
            *scan->counter = 0;
            const auto t0 = std::chrono::steady_clock::now();
            if (knn)
                scan->search_knn(queries, query_count, k, out);
            else
                scan->search_threshold(queries, query_count, correlation, out);
            return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
        catch (const std::exception &)
        {
            return -1.0;
        }
    }

    void tmref_sss_destroy(void *handle) { delete static_cast<SkipSequentialScan *>(handle); }

    // The reference's iSAX lower bound (SkipSequentialScan::lower_bound, the same bound as
    // TREMOR's record-level check, SkipSequential.cpp:200-211) of one raw template against every
    // owned window of a scan built with lower bounds: the number of windows whose bound does
    // not exceed `bound` (the windows a skip-sequential scan must still compute), and per block
    // of `block` consecutive windows whether any of them is such a window. For measuring how
    // much a lower-bound skip could prune; the scan's own statistics are not needed.
    int tmref_sss_lb_pass(void *handle, const float *query_raw, float bound, uint64_t block, uint8_t *any_pass,
                          uint64_t *passing)
    {
        auto *scan = static_cast<SkipSequentialScan *>(handle);
        if (!scan->lower_bounds || block == 0)
            return -1;
        try
        {
            std::vector<ts_type> znorm, paa;
            std::vector<int> order;
            scan->prepare_query(query_raw, znorm, paa, order);
            const long long W = static_cast<long long>(scan->subsequences);
            const long long nb = (W + static_cast<long long>(block) - 1) / static_cast<long long>(block);
            unsigned long long count = 0;
#pragma omp parallel for reduction(+ : count) schedule(static) num_threads(scan->threads)
            for (long long b = 0; b < nb; b++)
            {
                uint8_t any = 0;
                const long long end = std::min(W, (b + 1) * static_cast<long long>(block));
                for (long long id = b * static_cast<long long>(block); id < end; id++)
                {
                    if (scan->raw[id] == TREMOR_MISSING_VALUE)
                        continue;
                    if (scan->lower_bound(paa.data(), id) <= bound)
                    {
                        count++;
                        any = 1;
                    }
                }
                any_pass[b] = any;
            }
            *passing = count;
            return 0;
        }
        catch (const std::exception &)
        {
            return -1;
        }
    }

    // A sequential-mode scan (no lower bounds) over a record held in memory, with the
    // per-window statistics given instead of computed by build(): the members build() sets
    // for one rank (SkipSequential.cpp:138-163: window, first and count of the owned
    // subsequences, raw samples, means, stds) are assigned directly. For records of
    // 2^26-2^28 samples, where build()'s two-pass statistics (one dependent chain of m
    // FP64 additions per window) take minutes; the statistics given are the oracle's
    // restatement of them, pinned bit for bit to build()'s by the tests. The searches are
    // then the reference's own (search_knn / search_threshold via tmref_sss_search).
    void *tmref_sss_from_stats(const float *raw, uint64_t n, int m, const float *means, const float *stds,
                               int merge_offset, int threads)
    {
        try
        {
            const uint64_t W = n - static_cast<uint64_t>(m) + 1;
            auto *scan = new SkipSequentialScan(threads, 8, merge_offset, 0, false);
            scan->window = m;
            scan->first_subsequence = 0;
            scan->subsequences = static_cast<idx_t>(W);
            scan->raw.assign(raw, raw + n);
            scan->means.assign(means, means + W);
            scan->stds.assign(stds, stds + W);
            return scan;
        }
        catch (const std::exception &)
        {
            return nullptr;
        }
    }

    // The reference's FP32 distance (l2_dist_znorm_subsequence, no abandoning) of one raw
    // template against the windows at `positions`, with the scan's statistics and its own
    // template preparation (prepare_query: znormalize_inplace, query_block_order); -1 for a
    // window whose first sample is missing (not searched).
    int tmref_sss_distances(void *handle, const float *query_raw, const uint64_t *positions, uint64_t count,
                            float *out)
    {
        auto *scan = static_cast<SkipSequentialScan *>(handle);
        try
        {
            std::vector<ts_type> znorm, paa;
            std::vector<int> order;
            scan->prepare_query(query_raw, znorm, paa, order);
            for (uint64_t i = 0; i < count; i++)
            {
                const uint64_t id = positions[i] - static_cast<uint64_t>(scan->first_subsequence);
                if (id >= static_cast<uint64_t>(scan->subsequences))
                    return -1;
                if (scan->raw[id] == TREMOR_MISSING_VALUE)
                {
                    out[i] = -1.0f;
                    continue;
                }
                int blocks = 0;
                out[i] = l2_dist_znorm_subsequence(znorm.data(), scan->raw.data(), id, scan->window, scan->means[id],
                                                   scan->stds[id], FLT_MAX, order.data(), &blocks);
            }
            return 0;
        }
        catch (const std::exception &)
        {
            return -1;
        }
    }

    float tmref_l2_dist(const float *query_znorm, const float *raw, uint64_t start, int m, float mean, float stddev,
                        float bound, const int *block_order, int *blocks_visited)
    {
        return l2_dist_znorm_subsequence(query_znorm, raw, start, m, mean, stddev, bound, block_order, blocks_visited);
    }

    void tmref_znormalize(float *values, int len) { znormalize_inplace(values, len); }

    void tmref_block_order(const float *query_znorm, int m, int *order)
    {
        const std::vector<int> o = query_block_order(query_znorm, m);
        std::memcpy(order, o.data(), o.size() * sizeof(int));
    }

    float tmref_cc_to_ed(float cc, int m) { return cc_to_ed(cc, m); }
    float tmref_ed_to_cc(float ed, int m) { return ed_to_cc(ed, m); }

    // Canonical exclusion selection (ZnormSearch.hpp:170-189); returns the number kept.
    int tmref_select_knn(const uint64_t *positions, const float *distances, uint64_t count, int k, int merge_offset,
                         uint64_t *out_positions, float *out_distances)
    {
        std::vector<KnnCandidate> c(count);
        for (uint64_t i = 0; i < count; i++)
            c[i] = {positions[i], distances[i]};
        const std::vector<KnnCandidate> kept = select_knn_with_exclusion(c, k, merge_offset);
        for (size_t i = 0; i < kept.size(); i++)
        {
            out_positions[i] = kept[i].first;
            out_distances[i] = kept[i].second;
        }
        return static_cast<int>(kept.size());
    }

    // Exclusion-zone bound queue (iSAXPqueue.cpp:471-520): offers (distance, position)
    // pairs in order and returns the final queue contents.
    void tmref_pqueue_offset(const float *distances, const uint64_t *positions, uint64_t count, int size,
                             int merge_offset, float *out_knn, int64_t *out_positions)
    {
        pqueue_bsf *q = pqueue_bsf_init(size);
        for (uint64_t i = 0; i < count; i++)
            if (distances[i] < q->knn[size - 1])
                pqueue_bsf_insert_offset(q, distances[i], positions[i], nullptr, merge_offset);
        for (int i = 0; i < size; i++)
        {
            out_knn[i] = q->knn[i];
            out_positions[i] = q->position[i];
        }
        pqueue_bsf_destroy(q);
    }
}
