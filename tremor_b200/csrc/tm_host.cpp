// Host-side steps of the scan whose floating-point results must be bit-identical to
// the reference: template z-normalisation and block order, the cc <-> ED conversions,
// and the canonical answer selection. Compiled with -ffp-contract=off; every fused
// multiply-add the reference's g++ -O2 -mfma build performs is written as std::fma.
#include "tm_host.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>

namespace tm_host {

float cc_to_ed(float cc, int m) { return 2.0f * static_cast<float>(m) * (1.0f - cc); } // ZnormSearch.hpp:23-26

float ed_to_cc(float ed, int m) { return 1.0f - (ed / (2.0f * static_cast<float>(m))); } // ZnormSearch.hpp:28-31

// ZnormSearch.hpp:33-62
void znormalize(float *values, int len)
{
    if (values == nullptr || len <= 0)
        return;
    double sum = 0.0, sum_sq = 0.0;
    for (int i = 0; i < len; i++)
    {
        const double v = static_cast<double>(values[i]);
        sum += v;
        sum_sq = std::fma(v, v, sum_sq);
    }
    const double mean = sum / static_cast<double>(len);
    double variance = std::fma(-mean, mean, sum_sq / static_cast<double>(len));
    if (variance < 0.0)
        variance = 0.0;
    const double stddev = std::sqrt(variance);
    if (stddev <= 1e-12)
    {
        for (int i = 0; i < len; i++)
            values[i] = 0.0f;
        return;
    }
    for (int i = 0; i < len; i++)
        values[i] = static_cast<float>((static_cast<double>(values[i]) - mean) / stddev);
}

// ZnormSearch.hpp:72-90
void block_order(const float *q, int m, int *order)
{
    const int blocks = m / kZnormBlock;
    std::vector<std::pair<float, int>> energy(static_cast<size_t>(blocks));
    for (int b = 0; b < blocks; b++)
    {
        float e = 0.0f;
        for (int i = b * kZnormBlock; i < (b + 1) * kZnormBlock; i++)
            e = std::fma(q[i], q[i], e);
        energy[static_cast<size_t>(b)] = {e, b * kZnormBlock};
    }
    std::stable_sort(energy.begin(), energy.end(),
                     [](const std::pair<float, int> &a, const std::pair<float, int> &b) { return a.first > b.first; });
    for (int b = 0; b < blocks; b++)
        order[b] = energy[static_cast<size_t>(b)].second;
}

// ZnormSearch.hpp:170-189, over candidates sorted here by (distance, position).
int select_knn(std::vector<Hit> &cands, int k, int merge, std::vector<Hit> &kept)
{
    std::sort(cands.begin(), cands.end(), [](const Hit &a, const Hit &b) {
        return a.dist != b.dist ? a.dist < b.dist : a.pos < b.pos;
    });
    return extend_knn(cands, k, merge, kept);
}

// Greedy continuation: offers cands (already in (distance, position) order) to `kept`.
int extend_knn(const std::vector<Hit> &cands, int k, int merge, std::vector<Hit> &kept)
{
    for (const Hit &c : cands)
    {
        if (static_cast<int>(kept.size()) >= k)
            break;
        bool ok = true;
        for (const Hit &h : kept)
        {
            const uint64_t gap = c.pos > h.pos ? c.pos - h.pos : h.pos - c.pos;
            if (gap < static_cast<uint64_t>(merge))
            {
                ok = false;
                break;
            }
        }
        if (ok)
            kept.push_back(c);
    }
    return static_cast<int>(kept.size());
}

// SkipSequential.cpp:358-370 (= Tremor.cpp:2762-2793): by position, keep the first of
// detections closer than merge_offset + 1 to the last kept one.
void threshold_merge(std::vector<Hit> &hits, int merge, std::vector<Hit> &out)
{
    std::sort(hits.begin(), hits.end(), [](const Hit &a, const Hit &b) {
        return a.pos != b.pos ? a.pos < b.pos : a.dist < b.dist;
    });
    bool has_last = false;
    uint64_t last = 0;
    for (const Hit &h : hits)
    {
        if (has_last && h.pos == last)
            continue; // a window found twice is reported once (Tremor.cpp:2770-2775)
        if (has_last && merge > 0 && h.pos < last + static_cast<uint64_t>(merge + 1))
            continue;
        out.push_back(h);
        last = h.pos;
        has_last = true;
    }
}

} // namespace tm_host
