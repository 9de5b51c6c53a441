/*
 * tm_oracle — CPU restatement of TREMOR's exact scan path (TEST INFRASTRUCTURE).
 *
 * This library is the checker for the GPU product: only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline leg of bench.py may load it.
 * The product library (tremor_b200) never links, loads or calls it.
 *
 * Every function restates one reference function in plain C, in the same
 * floating-point operation order, so that its FP32 results are bit-identical to
 * the reference compiled with g++ -O2 -mavx2 -mfma (which contracts a*b+c into
 * fused multiply-adds). Citations are paths inside the reference project.
 *
 * Parity pins: tests/test_oracle.py checks these functions bit-for-bit against
 * the reference's own code built by `make -C oracle ref`, and against the
 * committed golden fixtures of tests/golden/ (a restatement of
 * experiments/validate_search.py's seeded case, answers produced by that build).
 */
#ifndef TM_ORACLE_H
#define TM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TMO_MISSING_VALUE (-100000.0f) /* ZnormSearch.hpp:21 */
#define TMO_ZNORM_BLOCK 32             /* ZnormSearch.hpp:65 */

/* ZnormSearch.hpp:23-31 */
float tmo_cc_to_ed(float cc, int m);
float tmo_ed_to_cc(float ed, int m);

/* ZnormSearch.hpp:33-62: FP64 one-pass z-normalisation, written back as float. */
void tmo_znormalize(float *values, int len);

/* ZnormSearch.hpp:72-90: whole 32-sample blocks by decreasing energy (stable). */
void tmo_block_order(const float *query_znorm, int m, int *order);

/* SkipSequential.cpp:157-190 (= indexing.cpp:128-152): exact two-pass FP64 mean and
 * population std of every window, stored as float; missing samples count as 0;
 * std <= 1e-12 -> 0; a window whose first sample is missing gets (0, 0). */
void tmo_window_stats(const float *raw, uint64_t windows, int m, float *mean, float *stddev);
/* The same statistics, bit for bit, 16 windows per vectorised pass (AVX2 + FMA hosts):
 * for records of 2^26-2^28 samples. */
void tmo_window_stats_fast(const float *raw, uint64_t windows, int m, float *mean, float *stddev);

/* ZnormSearch.hpp:103-165: z-normalised squared ED with block early abandoning. */
float tmo_l2_dist(const float *query_znorm, const float *raw, uint64_t start, int m, float mean, float stddev,
                  float bound, const int *block_order, int *blocks_visited);

/* ZnormSearch.hpp:170-189: canonical exclusion selection. Sorts the candidates in place
 * by (distance, position) and returns how many were kept (<= k). */
int tmo_select_knn(uint64_t *positions, float *distances, uint64_t count, int k, int merge_offset,
                   uint64_t *out_positions, float *out_distances);

/* Distance of every window of one raw template (z-normalised here): FLT_MAX for constant
 * windows, NaN-free; windows whose first sample is missing get -1 (not searched). */
void tmo_distance_profile(const float *raw, uint64_t n, int m, const float *query_raw, float *out);

/* SkipSequentialScan::search_knn (SkipSequential.cpp:376-473) on one rank, no lower bounds:
 * I/D are query_count x k, unfilled slots (0, FLT_MAX). Returns 0. */
int tmo_scan_knn(const float *raw, uint64_t n, int m, const float *queries, int query_count, int k, int merge_offset,
                 uint64_t *I, float *D);

/* SkipSequentialScan::search_threshold (SkipSequential.cpp:303-374) on one rank: hits in
 * output order (query, then position, merged). Returns the number of hits; writes at most
 * `capacity` of them. */
int64_t tmo_scan_threshold(const float *raw, uint64_t n, int m, const float *queries, int query_count,
                           float correlation, int merge_offset, int32_t *query_ids, uint64_t *positions,
                           float *distances, int64_t capacity);

#ifdef __cplusplus
}
#endif

#endif
