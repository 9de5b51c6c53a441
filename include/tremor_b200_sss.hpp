// GpuSkipSequentialScan: a drop-in for the reference's SkipSequentialScan
// (tremor/algos/sss/SkipSequential.hpp:32-78) on one B200, header-only over the C ABI
// of tremor_b200.h. Same constructor arguments, same build / search_threshold /
// search_knn calls, same output files and formats:
//   search_threshold -> <output>_<rank>.csv  "Query, Counter, Position, Cross Correlation"
//                       (SkipSequential.cpp:310-370)
//   search_knn       -> <output>             "tID, k, pos, corr" (SkipSequential.cpp:458-470)
// with the same answers. One process and one GPU: rank 0, one replication group, the
// whole waveform as the single data partition. lower_bounds only selects the label
// printed per template ("sss" / "ss"); the GPU scan computes every window exactly
// either way, which gives the same answers as skipping by iSAX lower bounds.
// Errors throw std::runtime_error, as the reference does for I/O failures.
#ifndef TREMOR_B200_SSS_HPP
#define TREMOR_B200_SSS_HPP

#include <cfloat>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "tremor_b200.h"

class GpuSkipSequentialScan
{
public:
    GpuSkipSequentialScan(int threads, int paa_segments, int merge_offset, int replication_groups,
                          bool lower_bounds = true, int device = 0)
        : merge_offset(merge_offset), lower_bounds(lower_bounds), device(device)
    {
        (void)threads;
        (void)paa_segments;
        if (replication_groups > 1)
            throw std::invalid_argument("--replication-groups must be between 0 and the number of ranks");
    }
    ~GpuSkipSequentialScan() { tm_ctx_destroy(ctx); }
    GpuSkipSequentialScan(const GpuSkipSequentialScan &) = delete;
    GpuSkipSequentialScan &operator=(const GpuSkipSequentialScan &) = delete;

    // Loads the waveform and computes the window statistics on the GPU.
    void build(const std::string &filename, uint64_t total_samples, int window_length)
    {
        window = window_length;
        std::vector<float> raw(total_samples);
        FILE *f = std::fopen(filename.c_str(), "rb");
        if (f == nullptr || std::fread(raw.data(), sizeof(float), raw.size(), f) != raw.size())
        {
            if (f)
                std::fclose(f);
            throw std::runtime_error("cannot read " + filename);
        }
        std::fclose(f);
        build(raw.data(), total_samples, window_length);
    }

    void build(const float *raw, uint64_t total_samples, int window_length)
    {
        window = window_length;
        tm_ctx_destroy(ctx);
        ctx = nullptr;
        check(tm_ctx_create(raw, total_samples, device, &ctx), "tm_ctx_create");
        check(tm_prepare_length(ctx, window), "tm_prepare_length");
        summary_bytes = static_cast<double>(total_samples - window + 1) * 9.0;
    }

    void search_threshold(const float *queries, int query_count, float correlation, const std::string &output)
    {
        FILE *out = std::fopen((output + "_0.csv").c_str(), "w");
        if (out == nullptr)
            throw std::runtime_error("cannot write threshold output " + output);
        std::fprintf(out, "Query, Counter, Position, Cross Correlation\n");
        const auto t0 = std::chrono::steady_clock::now();
        tm_result *res = nullptr;
        check(tm_search_threshold(ctx, queries, query_count, window, correlation, merge_offset, &res),
              "tm_search_threshold");
        for (int q = 0; q < query_count; q++)
        {
            uint64_t n = 0;
            tm_result_count(res, q, &n);
            std::vector<uint64_t> pos(n);
            std::vector<float> dist(n);
            tm_result_get(res, q, pos.data(), dist.data(), n);
            for (uint64_t c = 0; c < n; c++)
                std::fprintf(out, "%d, %lld, %llu, %f\n", q, static_cast<long long>(c),
                             static_cast<unsigned long long>(pos[c]), tm_ed_to_cc(dist[c], window));
        }
        tm_result_free(res);
        std::fclose(out);
        report(t0, query_count);
    }

    // Writes the kNN CSV; I_out / D_out (optional) receive the answers (query-major, k each).
    void search_knn(const float *queries, int query_count, int k, const std::string &output,
                    std::vector<uint64_t> *I_out = nullptr, std::vector<float> *D_out = nullptr)
    {
        std::vector<uint64_t> I(static_cast<size_t>(query_count) * k);
        std::vector<float> D(I.size());
        const auto t0 = std::chrono::steady_clock::now();
        check(tm_search_knn(ctx, queries, query_count, window, k, merge_offset, I.data(), D.data()), "tm_search_knn");
        FILE *out = std::fopen(output.c_str(), "w");
        if (out == nullptr)
            throw std::runtime_error("cannot write kNN output " + output);
        std::fprintf(out, "tID, k, pos, corr\n");
        for (int q = 0; q < query_count; q++)
            for (int j = 0; j < k; j++)
                std::fprintf(out, "%d, %d, %llu, %f\n", q, j + 1,
                             static_cast<unsigned long long>(I[static_cast<size_t>(q) * k + j]),
                             tm_ed_to_cc(D[static_cast<size_t>(q) * k + j], window));
        std::fclose(out);
        report(t0, query_count);
        if (I_out)
            *I_out = I;
        if (D_out)
            *D_out = D;
    }

    double summary_memory_bytes() const { return summary_bytes; }

private:
    void check(int rc, const char *what) const
    {
        if (rc != TM_OK)
            throw std::runtime_error(std::string(what) + " failed (" + std::to_string(rc) + "): " +
                                     (ctx ? tm_last_error(ctx) : ""));
    }
    void report(std::chrono::steady_clock::time_point t0, int queries) const
    {
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("[Node 0] %d queries: %.6f s (%s, gpu)\n", queries, s, lower_bounds ? "sss" : "ss");
    }

    tm_ctx *ctx = nullptr;
    int merge_offset = 0;
    bool lower_bounds = true;
    int device = 0;
    int window = 0;
    double summary_bytes = 0.0;
};

#endif
