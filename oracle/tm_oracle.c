/*
 * tm_oracle.c — CPU restatement of TREMOR's exact scan path. TEST INFRASTRUCTURE:
 * the GPU product never links or calls this file (see tm_oracle.h).
 *
 * Compiled with -ffp-contract=off: every fused multiply-add below is written out
 * with fma()/fmaf() where the reference, built with g++ -O2 -mfma (GCC contracts
 * C++ floating-point expressions by default), computes one. The choice of each
 * fusion is pinned bit-for-bit against the reference build in tests/test_oracle.py.
 */
#include "tm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

float tmo_cc_to_ed(float cc, int m) { return 2.0f * (float)m * (1.0f - cc); }

float tmo_ed_to_cc(float ed, int m) { return 1.0f - (ed / (2.0f * (float)m)); }

void tmo_znormalize(float *values, int len)
{
    if (values == NULL || len <= 0)
        return;
    double sum = 0.0, sum_sq = 0.0;
    for (int i = 0; i < len; i++)
    {
        const double v = (double)values[i];
        sum += v;
        sum_sq = fma(v, v, sum_sq);
    }
    const double mean = sum / (double)len;
    double variance = fma(-mean, mean, sum_sq / (double)len);
    if (variance < 0.0)
        variance = 0.0;
    const double stddev = sqrt(variance);
    if (stddev <= 1e-12)
    {
        for (int i = 0; i < len; i++)
            values[i] = 0.0f;
        return;
    }
    for (int i = 0; i < len; i++)
        values[i] = (float)(((double)values[i] - mean) / stddev);
}

void tmo_block_order(const float *q, int m, int *order)
{
    const int blocks = m / TMO_ZNORM_BLOCK;
    float *energy = (float *)malloc(sizeof(float) * (size_t)(blocks > 0 ? blocks : 1));
    for (int b = 0; b < blocks; b++)
    {
        float e = 0.0f;
        for (int i = b * TMO_ZNORM_BLOCK; i < (b + 1) * TMO_ZNORM_BLOCK; i++)
            e = fmaf(q[i], q[i], e);
        energy[b] = e;
        order[b] = b;
    }
    /* stable insertion sort by decreasing energy (std::stable_sort with a > comparator) */
    for (int i = 1; i < blocks; i++)
    {
        const int id = order[i];
        const float e = energy[id];
        int j = i - 1;
        while (j >= 0 && energy[order[j]] < e)
        {
            order[j + 1] = order[j];
            j--;
        }
        order[j + 1] = id;
    }
    for (int b = 0; b < blocks; b++)
        order[b] *= TMO_ZNORM_BLOCK;
    free(energy);
}

static inline double clean64(float v) { return v == TMO_MISSING_VALUE ? 0.0 : (double)v; }

void tmo_window_stats(const float *raw, uint64_t windows, int m, float *mean_out, float *std_out)
{
#pragma omp parallel for schedule(static)
    for (long long id = 0; id < (long long)windows; id++)
    {
        const float *w = raw + id;
        if (w[0] == TMO_MISSING_VALUE)
        {
            mean_out[id] = 0.0f;
            std_out[id] = 0.0f;
            continue;
        }
        double sum = 0.0;
        for (int d = 0; d < m; d++)
            sum += clean64(w[d]);
        const double mean = sum / m;
        double squares = 0.0;
        for (int d = 0; d < m; d++)
        {
            const double v = clean64(w[d]) - mean;
            squares = fma(v, v, squares);
        }
        const double stddev = sqrt(squares / m);
        mean_out[id] = (float)mean;
        std_out[id] = (float)(stddev <= 1e-12 ? 0.0 : stddev);
    }
}

/* tmo_window_stats for records of any size: the same per-window operations in the same
 * order (SkipSequential.cpp:157-190: a sequential FP64 sum, the mean, a sequential FP64 sum
 * of fused squares), for 32 consecutive windows at once. Sample t (relative to the block's
 * first window) is the (t - j)-th term of window j, so walking the samples in order and
 * adding each one to every window that contains it gives every window its terms in the
 * reference's order; in the middle of the walk all 32 windows take the same sample, a
 * broadcast that vectorises (AVX2 + FMA, which every host of the reference build has).
 * The results are those of tmo_window_stats bit for bit (checked by tests/test_oracle.py).
 * The reference's build() runs one window per thread, a dependent chain of m additions;
 * at 2^28 samples and m = 4096 this form takes seconds where that takes minutes. */
#define TMO_STATS_BLOCK 32

typedef double tmo_v4d __attribute__((vector_size(32))); /* 4 windows' sums, one AVX2 register */

__attribute__((target("avx2,fma"))) static void stats_block(const float *w, int m, double *mean, double *sd)
{
    double sum[TMO_STATS_BLOCK] = {0}, sq[TMO_STATS_BLOCK] = {0};
    const int B = TMO_STATS_BLOCK, last = m + B - 1; /* samples t in [0, last) */
    /* ramp-in (t < B - 1): windows 0..t; the full middle: all B windows (eight registers);
     * ramp-out (t >= m): windows t - m + 1..B - 1 */
    const int mid_lo = B - 1, mid_hi = m; /* t in [mid_lo, mid_hi) takes every window */
    for (int t = 0; t < (mid_lo < last ? mid_lo : last); t++)
    {
        const double v = clean64(w[t]);
        for (int j = (t - m + 1 > 0 ? t - m + 1 : 0); j <= t; j++)
            sum[j] += v;
    }
    if (mid_lo < mid_hi)
    {
        tmo_v4d s[8];
        memcpy(s, sum, sizeof(s));
        for (int t = mid_lo; t < mid_hi; t++)
        {
            const double v = clean64(w[t]);
            const tmo_v4d vv = {v, v, v, v};
#pragma GCC unroll 8
            for (int r = 0; r < 8; r++)
                s[r] += vv;
        }
        memcpy(sum, s, sizeof(s));
    }
    for (int t = (mid_hi > mid_lo ? mid_hi : mid_lo); t < last; t++)
    {
        const double v = clean64(w[t]);
        const int jlo = t - m + 1 > 0 ? t - m + 1 : 0, jhi = t < B - 1 ? t : B - 1;
        for (int j = jlo; j <= jhi; j++)
            sum[j] += v;
    }
    for (int j = 0; j < B; j++)
        mean[j] = sum[j] / m;
    for (int t = 0; t < (mid_lo < last ? mid_lo : last); t++)
    {
        const double v = clean64(w[t]);
        for (int j = (t - m + 1 > 0 ? t - m + 1 : 0); j <= t; j++)
        {
            const double d = v - mean[j];
            sq[j] = fma(d, d, sq[j]);
        }
    }
    if (mid_lo < mid_hi)
    {
        tmo_v4d q[8], mu[8];
        memcpy(q, sq, sizeof(q));
        memcpy(mu, mean, sizeof(mu));
        for (int t = mid_lo; t < mid_hi; t++)
        {
            const double v = clean64(w[t]);
            const tmo_v4d vv = {v, v, v, v};
#pragma GCC unroll 8
            for (int r = 0; r < 8; r++)
            {
                const tmo_v4d d = vv - mu[r];
                q[r] = __builtin_ia32_vfmaddpd256(d, d, q[r]); /* fused, as fma() */
            }
        }
        memcpy(sq, q, sizeof(q));
    }
    for (int t = (mid_hi > mid_lo ? mid_hi : mid_lo); t < last; t++)
    {
        const double v = clean64(w[t]);
        const int jlo = t - m + 1 > 0 ? t - m + 1 : 0, jhi = t < B - 1 ? t : B - 1;
        for (int j = jlo; j <= jhi; j++)
        {
            const double d = v - mean[j];
            sq[j] = fma(d, d, sq[j]);
        }
    }
    for (int j = 0; j < B; j++)
        sd[j] = sqrt(sq[j] / m);
}

void tmo_window_stats_fast(const float *raw, uint64_t windows, int m, float *mean_out, float *std_out)
{
    const long long blocks = (long long)(windows / TMO_STATS_BLOCK);
#pragma omp parallel for schedule(dynamic, 64)
    for (long long b = 0; b < blocks; b++)
    {
        const uint64_t id0 = (uint64_t)b * TMO_STATS_BLOCK;
        const float *w = raw + id0;
        double mean[TMO_STATS_BLOCK], sd[TMO_STATS_BLOCK];
        stats_block(w, m, mean, sd);
        for (int j = 0; j < TMO_STATS_BLOCK; j++)
        {
            const uint64_t id = id0 + (uint64_t)j;
            if (w[j] == TMO_MISSING_VALUE)
            {
                mean_out[id] = 0.0f;
                std_out[id] = 0.0f;
                continue;
            }
            mean_out[id] = (float)mean[j];
            std_out[id] = (float)(sd[j] <= 1e-12 ? 0.0 : sd[j]);
        }
    }
    const uint64_t done = (uint64_t)blocks * TMO_STATS_BLOCK;
    if (done < windows)
        tmo_window_stats(raw + done, windows - done, m, mean_out + done, std_out + done);
}

/* hsum256 (ZnormSearch.hpp:92-97) of the lane-wise sum acc0 + acc1. */
static inline float hsum16(const float *acc0, const float *acc1)
{
    float v[8];
    for (int l = 0; l < 8; l++)
        v[l] = acc0[l] + acc1[l];
    const float s0 = v[0] + v[4], s1 = v[1] + v[5], s2 = v[2] + v[6], s3 = v[3] + v[7];
    return (s0 + s2) + (s1 + s3);
}

float tmo_l2_dist(const float *q, const float *raw_seq, uint64_t start, int m, float mean, float stddev, float bound,
                  const int *order, int *blocks_visited)
{
    if (q == NULL || raw_seq == NULL || m <= 0)
        return FLT_MAX;
    if (stddev <= 1e-12f)
        return FLT_MAX;
    const float *raw = raw_seq + start;
    const float inv_std = 1.0f / stddev;
    float acc0[8] = {0}, acc1[8] = {0};
    const int blocks = m / TMO_ZNORM_BLOCK;
    for (int b = 0; b < blocks; b++)
    {
        const int off = order[b];
        for (int i = off; i < off + TMO_ZNORM_BLOCK; i += 16)
        {
            for (int l = 0; l < 8; l++)
            {
                float r0 = raw[i + l], r1 = raw[i + 8 + l];
                if (r0 == TMO_MISSING_VALUE)
                    r0 = 0.0f;
                if (r1 == TMO_MISSING_VALUE)
                    r1 = 0.0f;
                const float d0 = fmaf(-(r0 - mean), inv_std, q[i + l]);
                const float d1 = fmaf(-(r1 - mean), inv_std, q[i + 8 + l]);
                acc0[l] = fmaf(d0, d0, acc0[l]);
                acc1[l] = fmaf(d1, d1, acc1[l]);
            }
        }
        const float dist = hsum16(acc0, acc1);
        if (dist > bound)
        {
            *blocks_visited = b + 1;
            return dist;
        }
    }
    *blocks_visited = blocks;
    float dist = hsum16(acc0, acc1);
    for (int i = blocks * TMO_ZNORM_BLOCK; i < m; i++)
    {
        const float raw_v = raw[i] == TMO_MISSING_VALUE ? 0.0f : raw[i];
        const float diff = fmaf(-(raw_v - mean), inv_std, q[i]);
        dist = fmaf(diff, diff, dist);
    }
    return dist;
}

typedef struct
{
    uint64_t pos;
    float dist;
} cand_t;

static int cmp_dist_pos(const void *a, const void *b)
{
    const cand_t *x = (const cand_t *)a, *y = (const cand_t *)b;
    if (x->dist != y->dist)
        return x->dist < y->dist ? -1 : 1;
    return x->pos < y->pos ? -1 : (x->pos > y->pos ? 1 : 0);
}

static int cmp_pos_dist(const void *a, const void *b)
{
    const cand_t *x = (const cand_t *)a, *y = (const cand_t *)b;
    if (x->pos != y->pos)
        return x->pos < y->pos ? -1 : 1;
    return x->dist < y->dist ? -1 : (x->dist > y->dist ? 1 : 0);
}

/* greedy over candidates already sorted by (distance, position) */
static int greedy_exclusion(const cand_t *c, uint64_t count, int k, int merge, uint64_t *op, float *od)
{
    int kept = 0;
    for (uint64_t i = 0; i < count && kept < k; i++)
    {
        int ok = 1;
        for (int j = 0; j < kept; j++)
        {
            const uint64_t a = c[i].pos, b = op[j];
            const uint64_t gap = a > b ? a - b : b - a;
            if (gap < (uint64_t)merge)
            {
                ok = 0;
                break;
            }
        }
        if (!ok)
            continue;
        op[kept] = c[i].pos;
        od[kept] = c[i].dist;
        kept++;
    }
    return kept;
}

int tmo_select_knn(uint64_t *positions, float *distances, uint64_t count, int k, int merge_offset,
                   uint64_t *out_positions, float *out_distances)
{
    cand_t *c = (cand_t *)malloc(sizeof(cand_t) * (count ? count : 1));
    for (uint64_t i = 0; i < count; i++)
    {
        c[i].pos = positions[i];
        c[i].dist = distances[i];
    }
    qsort(c, count, sizeof(cand_t), cmp_dist_pos);
    for (uint64_t i = 0; i < count; i++)
    {
        positions[i] = c[i].pos;
        distances[i] = c[i].dist;
    }
    const int kept = greedy_exclusion(c, count, k, merge_offset, out_positions, out_distances);
    free(c);
    return kept;
}

void tmo_distance_profile(const float *raw, uint64_t n, int m, const float *query_raw, float *out)
{
    const uint64_t windows = n - (uint64_t)m + 1;
    float *q = (float *)malloc(sizeof(float) * (size_t)m);
    int *order = (int *)malloc(sizeof(int) * (size_t)(m / TMO_ZNORM_BLOCK + 1));
    float *mean = (float *)malloc(sizeof(float) * windows);
    float *sd = (float *)malloc(sizeof(float) * windows);
    memcpy(q, query_raw, sizeof(float) * (size_t)m);
    tmo_znormalize(q, m);
    tmo_block_order(q, m, order);
    tmo_window_stats(raw, windows, m, mean, sd);
#pragma omp parallel for schedule(static)
    for (long long j = 0; j < (long long)windows; j++)
    {
        int blocks = 0;
        out[j] = raw[j] == TMO_MISSING_VALUE ? -1.0f
                                             : tmo_l2_dist(q, raw, (uint64_t)j, m, mean[j], sd[j], FLT_MAX, order, &blocks);
    }
    free(q);
    free(order);
    free(mean);
    free(sd);
}

int tmo_scan_knn(const float *raw, uint64_t n, int m, const float *queries, int query_count, int k, int merge_offset,
                 uint64_t *I, float *D)
{
    const uint64_t windows = n - (uint64_t)m + 1;
    float *prof = (float *)malloc(sizeof(float) * windows);
    cand_t *c = (cand_t *)malloc(sizeof(cand_t) * windows);
    for (int qi = 0; qi < query_count; qi++)
    {
        tmo_distance_profile(raw, n, m, queries + (size_t)qi * m, prof);
        uint64_t count = 0;
        for (uint64_t j = 0; j < windows; j++)
            if (prof[j] >= 0.0f)
            {
                c[count].pos = j;
                c[count].dist = prof[j];
                count++;
            }
        qsort(c, count, sizeof(cand_t), cmp_dist_pos);
        uint64_t *ip = I + (size_t)qi * k;
        float *dp = D + (size_t)qi * k;
        const int kept = greedy_exclusion(c, count, k, merge_offset, ip, dp);
        for (int j = kept; j < k; j++)
        {
            ip[j] = 0;
            dp[j] = FLT_MAX;
        }
    }
    free(prof);
    free(c);
    return 0;
}

int64_t tmo_scan_threshold(const float *raw, uint64_t n, int m, const float *queries, int query_count,
                           float correlation, int merge_offset, int32_t *query_ids, uint64_t *positions,
                           float *distances, int64_t capacity)
{
    const uint64_t windows = n - (uint64_t)m + 1;
    const float bound = tmo_cc_to_ed(correlation, m);
    float *prof = (float *)malloc(sizeof(float) * windows);
    cand_t *c = (cand_t *)malloc(sizeof(cand_t) * windows);
    int64_t total = 0;
    for (int qi = 0; qi < query_count; qi++)
    {
        tmo_distance_profile(raw, n, m, queries + (size_t)qi * m, prof);
        uint64_t count = 0;
        for (uint64_t j = 0; j < windows; j++)
            if (prof[j] >= 0.0f && prof[j] <= bound)
            {
                c[count].pos = j;
                c[count].dist = prof[j];
                count++;
            }
        qsort(c, count, sizeof(cand_t), cmp_pos_dist);
        int has_last = 0;
        uint64_t last = 0;
        for (uint64_t i = 0; i < count; i++)
        {
            if (has_last && merge_offset > 0 && c[i].pos < last + (uint64_t)(merge_offset + 1))
                continue;
            if (total < capacity)
            {
                query_ids[total] = qi;
                positions[total] = c[i].pos;
                distances[total] = c[i].dist;
            }
            total++;
            last = c[i].pos;
            has_last = 1;
        }
    }
    free(prof);
    free(c);
    return total;
}
