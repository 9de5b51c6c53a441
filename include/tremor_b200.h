/*
 * tremor_b200 — C ABI of the B200 exact template-matching scan.
 *
 * One context holds one single-channel float32 waveform resident on one GPU,
 * plus per-template-length window statistics. Every search returns exactly the
 * answer sets of TREMOR's exact scan (the sequential / skip-sequential scan and
 * the scan and FFT branches of the adaptive planner): the same kNN answers with
 * the same exclusion-zone rule, the same threshold hits after the same merge,
 * and bit-identical FP32 distances.
 *
 * Conventions
 *   - every function returns int: TM_OK (0) or a negative TM_ERR_* code; nothing
 *     exits or throws across this boundary; tm_last_error() describes the last
 *     failure of a context;
 *   - host buffers are caller-owned; device buffers are owned by the library;
 *   - positions are window start indices into the whole waveform (uint64),
 *     distances are squared z-normalised Euclidean distances (FP32),
 *     ED^2 = 2 m (1 - correlation) (ZnormSearch.hpp:23-31);
 *   - a context may be used by one host thread at a time.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   tm_ctx_create + tm_prepare_length  <- SkipSequentialScan::build
 *        (tremor/algos/sss/SkipSequential.hpp:42; stats SkipSequential.cpp:157-190)
 *        and Tremor::buildIndexLongSequence (tremor/algos/htremor/Tremor.hpp:168-169;
 *        stats tremor/algos/tremor/indexing.cpp:128-152)
 *   tm_search_knn        <- SkipSequentialScan::search_knn (SkipSequential.hpp:48) and
 *                           Tremor::searchIndex in kNN mode (Tremor.hpp:172)
 *   tm_search_threshold  <- SkipSequentialScan::search_threshold (SkipSequential.hpp:45)
 *                           and Tremor::searchIndex in threshold mode
 *   tm_scan_batch        <- the per-template scan/FFT branches of the planner,
 *                           refine_in_position_order / fft_in_position_order
 *                           (tremor/algos/tremor/Tremor.cpp:1946, :2088), many
 *                           templates (of any lengths and modes) per call
 */
#ifndef TREMOR_B200_H
#define TREMOR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TM_OK 0
#define TM_ERR_ARGUMENT (-1)  /* invalid argument (sizes, null pointers, m > n) */
#define TM_ERR_CUDA (-2)      /* a CUDA call failed; see tm_last_error */
#define TM_ERR_NO_MEMORY (-3) /* device or host allocation failed */
#define TM_ERR_STATE (-4)     /* call not valid in the context's state */
#define TM_ERR_CAPACITY (-5)  /* caller buffer too small; the needed size was written */
#define TM_ERR_NO_DEVICE (-6) /* no usable sm_100 device */
#define TM_ERR_TIMEOUT (-7)   /* a kernel gave up waiting (bounded wait); the context stays usable */
#define TM_ERR_TOO_LARGE (-8) /* input larger than the fixed scratch of tm_window_stats_noalloc */

/* TREMOR_MISSING_VALUE (ZnormSearch.hpp:21): a missing sample counts as 0; a window
 * whose first sample is missing is not searched. */
#define TM_MISSING_VALUE (-100000.0f)

/* query modes, as Tremor::setModeKNN / setModeThreshold (Tremor.hpp:152-153) */
#define TM_MODE_THRESHOLD 0
#define TM_MODE_KNN 1

/* contraction kernels */
#define TM_KERNEL_AUTO 0       /* split-BF16 tensor cores where available, else FP32 */
#define TM_KERNEL_FP32 1       /* plain FP32 sliding dot product (CUDA cores) */
#define TM_KERNEL_SPLIT_BF16 2 /* tcgen05 split-BF16 Hankel contraction */

/* Tile shapes of the tensor-core contraction for batches of templates of several lengths
 * (tm_set_tiles). A tile's K extent is its longest template. Row tiles (k_scan_umma) hold
 * 128 templates x 256 windows; column tiles (k_scan_wm) hold 128 windows x 32, 64 or 128
 * templates, which wastes less when few templates share a length. AUTO picks the shape
 * of least modelled time per group (tm_autotune measures the model's constants). */
#define TM_TILES_AUTO 0
#define TM_TILES_ROWS 1
#define TM_TILES_COLS_128 2
#define TM_TILES_COLS_64 3
#define TM_TILES_COLS_32 4
/* Not a tile shape: the FP64 FFT branch (overlap-save correlation of each template with
 * the record, the same bounded epilogue and exact re-scoring), for few templates of up to
 * 16384 samples; its cost does not grow with the length. AUTO chooses it when the model
 * says it is faster than every tile shape. */
#define TM_TILES_FFT 5

/* request flags */
#define TM_FLAG_ZNORMALIZED 1u /* templ is already z-normalised (QaWorkerData::ts) */

typedef struct tm_ctx tm_ctx;
typedef struct tm_result tm_result;
typedef struct tm_batch tm_batch;

/* One template request (kNN or threshold). */
typedef struct tm_request
{
    const float *templ;    /* m samples, host memory */
    int32_t m;             /* template length (>= 1) */
    int32_t mode;          /* TM_MODE_KNN or TM_MODE_THRESHOLD */
    int32_t k;             /* kNN: answers wanted (>= 1) */
    int32_t merge_offset;  /* exclusion zone / threshold merge offset (>= 0) */
    float correlation;     /* threshold: minimum Pearson correlation */
    uint32_t flags;        /* TM_FLAG_* */
} tm_request;

/* ---- context ------------------------------------------------------------------ */

/* Copies the host waveform raw[0..n) to `device` and makes it resident. */
int tm_ctx_create(const float *raw, uint64_t n, int device, tm_ctx **out);
int tm_ctx_destroy(tm_ctx *ctx);
/* Text of the last error of this context ("" if none). */
const char *tm_last_error(const tm_ctx *ctx);
/* TM_KERNEL_*; default TM_KERNEL_AUTO. */
int tm_set_kernel(tm_ctx *ctx, int kernel);
/* Tile shape of mixed-length groups (TM_TILES_*); applies to batches created afterwards.
 * No counterpart in the reference (its scan has no tiles). */
int tm_set_tiles(tm_ctx *ctx, int tiles);
/* Tiling model of the planner behind TM_TILES_AUTO: kernel milliseconds of 128 templates x
 * 2^25 windows, [group kind: one length, several][shape: rows, columns 128, 64, 32]
 * [K: 256, 1024, 4096, 16384], 32 doubles in that order, then the FFT branch's
 * milliseconds per template per 2^25 samples for templates of up to 8192 samples and for
 * longer ones. tm_autotune measures it on this device (a few seconds, its own synthetic
 * record), stores it in the context and copies it to ms (up to capacity values); returns 34
 * or an error. tm_set_tile_model installs a saved one (count 34; 33 keeps the long-template
 * FFT figure, 32 both). No counterpart in the reference. */
int tm_autotune(tm_ctx *ctx, double *ms, int capacity);
int tm_set_tile_model(tm_ctx *ctx, const double *ms, int count);
/* Restricts searches to windows [first, first + count) (a data partition as in
 * SkipSequential.cpp:218-226); default: every window of every length. */
int tm_set_window_range(tm_ctx *ctx, uint64_t first, uint64_t count);
/* Computes (or reuses) the statistics of every window of length m. Optional: the
 * searches prepare the lengths they need. */
int tm_prepare_length(tm_ctx *ctx, int m);
/* The statistics the reference keeps per window (SkipSequential.hpp:74): float mean and
 * population std, (0, 0) for windows whose first sample is missing and std 0 for
 * constant windows. Bit-identical to the reference's two-pass FP64 values. Writes
 * count floats to each array, for windows [first, first + count). */
int tm_window_stats(tm_ctx *ctx, int m, uint64_t first, uint64_t count, float *mean, float *stddev);

/* ---- searches ------------------------------------------------------------------ */

/* kNN for `count` raw templates of length m (row-major count x m): I, D are count x k,
 * answers in order of (distance, position), unfilled slots (0, FLT_MAX) as the
 * reference's writers and Tremor::searchIndex (Tremor.cpp:3699-3718). */
int tm_search_knn(tm_ctx *ctx, const float *queries, int count, int m, int k, int merge_offset, uint64_t *I,
                  float *D);

/* Threshold search: every window with correlation >= `correlation`, merged by position
 * with the merge offset (SkipSequential.cpp:358-370). Results in *out. */
int tm_search_threshold(tm_ctx *ctx, const float *queries, int count, int m, float correlation, int merge_offset,
                        tm_result **out);

/* Any mix of kNN and threshold requests of any lengths in one call. */
int tm_scan_batch(tm_ctx *ctx, const tm_request *requests, int count, tm_result **out);

/* A batch prepared once (host z-normalisation, block orders, error-bound constants)
 * whose templates stay resident on the device; run it any number of times. The
 * serving loop and repeated searches of one template set use it; tm_scan_batch is
 * create + run + destroy. A batch belongs to the context that created it. */
int tm_batch_create(tm_ctx *ctx, const tm_request *requests, int count, tm_batch **out);
int tm_batch_run(tm_ctx *ctx, tm_batch *batch, tm_result **out);
int tm_batch_destroy(tm_batch *batch);
/* Host-to-device bytes tm_batch_create copied (templates, orders, constants). */
int tm_batch_h2d_bytes(const tm_batch *batch, uint64_t *bytes);

/* Results: per request, its answers (kNN: exactly k, padded; threshold: the merged hits). */
int tm_result_count(const tm_result *res, int request, uint64_t *count);
int tm_result_get(const tm_result *res, int request, uint64_t *positions, float *distances, uint64_t capacity);
void tm_result_free(tm_result *res);
/* The error of each answer against FP64. For the answers of request `request` of res (a
 * result of this context; the order of tm_result_get), writes min(count, capacity)
 * doubles: the squared z-normalised distance of the same template and window recomputed
 * entirely in FP64 from the raw samples (templ: the request's m template samples, raw or
 * already z-normalised, z-normalised again here in FP64 by two passes; the window's
 * two-pass FP64 mean and population std, missing samples counted as 0; an FP64 sum of
 * squared differences). Answers of distance FLT_MAX (kNN padding, constant windows) get
 * +inf. The relative error of answer i is |D_i - d64_i| / d64_i. No counterpart in the
 * reference, whose validation compares correlations with an FP64 implementation within
 * 2e-4 (experiments/validate_search.py:80-86, :127). */
int tm_result_fp64(tm_ctx *ctx, const tm_result *res, int request, const float *templ, int m, double *d64,
                   uint64_t capacity);

/* ---- allocation-free statistics ------------------------------------------------------ */

/* No counterpart in the reference: an entry point for callers that must not allocate
 * device memory (a live detector with a fixed latency budget, where cudaMalloc may
 * synchronise the device; a runtime whose pool allocator holds the free memory). It computes, on the calling thread's current device
 * and on `stream` (a cudaStream_t, 0 for the default stream), the statistics of every
 * window of length m of the device-resident waveform raw[0..n): mean, std and flags per
 * window into caller-owned device arrays of n - m + 1 elements, with the meaning of
 * tm_window_stats (equal to its values within a few float ulps) and flags bit 0 = first
 * sample missing, bit 1 = constant window, bit 3 = two-pass statistics. It allocates
 * nothing and does not synchronise: its only scratch is a fixed 8 MiB device array that
 * every GPU loading the library holds until the process exits, so n + m must not exceed
 * 524288 samples (larger inputs return TM_ERR_TOO_LARGE). The first call on a device
 * looks that array up on the device and keeps its address for the rest of the process
 * (make that first call before any stream capture; after cudaDeviceReset on that device
 * the kept address is stale, so do not call it again in that process). All calls share
 * the array: calls whose work overlaps on the GPU (other streams, other threads) race. */
int tm_window_stats_noalloc(const float *raw, uint64_t n, int m, float *mean, float *stddev, uint8_t *flags,
                            void *stream);

/* ---- conversions (ZnormSearch.hpp:23-31, bit-identical) -------------------------- */
float tm_cc_to_ed(float correlation, int m);
float tm_ed_to_cc(float distance, int m);

/* ---- instrumentation -------------------------------------------------------------- */

/* When enabled, the dominant contraction kernel is bracketed by CUDA events on the
 * library's stream and its launches and device time are accumulated. */
int tm_profile_enable(tm_ctx *ctx, int enable);
/* Name of the dominant kernel, its launch count, total device milliseconds, the
 * algorithmic flops it performed (2 m per template-window pair) and the number of
 * kernel launches of this library since the last reset. Resets the counters. */
int tm_profile_read(tm_ctx *ctx, char *name, size_t name_capacity, int64_t *launches, double *milliseconds,
                    double *flops, int64_t *all_launches);
/* Measured FP32 FMA rate of a device in TFLOP/s (2 flops per FMA; register-resident FMA
 * chains on every SM, best of 4 timed launches): the roofline denominator of the FP32
 * contraction kernel. No counterpart in the reference. */
int tm_fp32_peak(int device, double *tflops);
/* Milliseconds spent, since the last call and while profiling was enabled, in each of the
 * TM_PHASES phases of a search: [0] contraction kernel, [1] kNN bound, bucket list and
 * FP32 re-pass, [2] exact re-scoring, [3] answer filter and sort on the device, [4] copy
 * of the answers to the host, [5] answer selection on the host. Device phases are
 * CUDA-event spans on the context's stream. Writes min(capacity, TM_PHASES) values,
 * resets the counters, returns TM_PHASES. No counterpart in the reference (its searches
 * report wall-clock totals only). */
#define TM_PHASES 6
int tm_profile_phases(tm_ctx *ctx, double *milliseconds, int capacity);
/* Diagnostic: for `count` raw templates of length m, the contraction kernel's distance d
 * and error bound e of every (template, window) pair, and (if `exact` is not null) the
 * reference's exact FP32 distance of every pair; count x windows floats each, for the
 * context's window range. The bound holds when |d - exact| <= e (windows that are not
 * searched stay NaN in d and e). Small cases only: windows x count <= 2^31. */
int tm_bound_diagnostics(tm_ctx *ctx, const float *queries, int count, int m, float *d, float *e, float *exact);
/* One template, as the planner's worker seam calls the scan (Tremor.cpp:1946,
 * refine_in_position_order, one template per call). tm_scan_knn: the canonical kNN
 * answers of the context's windows (k entries in I/D, unfilled slots (0, FLT_MAX));
 * answers whose distance exceeds bound_in (the caller's current k-th distance; FLT_MAX
 * when it has none) are returned as (0, FLT_MAX), as the caller's queue would reject them
 * (offer_knn_window, Tremor.cpp:1352-1362). tm_scan_threshold: the merged threshold hits
 * (one request in *out). */
int tm_scan_knn(tm_ctx *ctx, const float *templ, int m, int k, int merge_offset, float bound_in, uint64_t *I,
                float *D);
int tm_scan_threshold(tm_ctx *ctx, const float *templ, int m, float correlation, int merge_offset,
                      tm_result **out);
/* Device-to-host bytes the searches of this context copied since the last call (resets). */
int tm_d2h_bytes(tm_ctx *ctx, uint64_t *bytes);
/* The context's CUDA stream (a cudaStream_t), for callers that order or time work on it. */
int tm_ctx_stream(tm_ctx *ctx, void **stream);
/* Candidates re-scored exactly in the last search (diagnostic). */
int tm_last_candidates(const tm_ctx *ctx, uint64_t *count);

/* ---- Serving: continuous batching over the resident waveform ----------------------
 * No counterpart in the reference, which hands template ids to MPI ranks
 * (Tremor.cpp:796-905, SkipSequential.cpp:97-136); this is the single-GPU equivalent.
 * tm_serve_start builds the resident FP64 prefix sums and starts `workers` threads, each
 * with its own stream and scratch. tm_submit queues one request (its template is copied;
 * any thread may submit). Each worker admits the oldest pending requests, at most
 * max_batch and within the device-memory budget for requests in flight, runs them as one
 * batch of mixed lengths and completes them; batches of different workers overlap on the
 * device. tm_poll returns completions (one consumer). Every request's answers equal those
 * of the same request searched alone. Lengths up to 16384; needs the tensor-core kernel.
 * While serving, tm_set_kernel and tm_set_window_range return TM_ERR_STATE; the other
 * calls stay usable. */
typedef struct tm_serve_config
{
    int workers;            /* batches in flight at once (1-8; default 1: on one GPU, concurrent
                             * batches mostly compete for the SMs and split the queue into
                             * smaller, less efficient batches) */
    int max_batch;          /* requests per batch at most (default 256) */
    uint64_t memory_budget; /* device bytes for requests in flight; 0: a quarter of the free memory */
    double batch_ms;        /* modelled device milliseconds of a batch at most (the planner's model,
                             * tm_autotune): admission stops there, so a request arriving during a
                             * batch waits for a bounded one; 0: no limit (a first request alone is
                             * always admitted) */
} tm_serve_config;

typedef struct tm_completion
{
    uint64_t ticket;   /* as returned by tm_submit */
    int status;        /* TM_OK, or the error of the batch that carried the request */
    int batch_size;    /* requests in that batch */
    tm_result *result; /* the request's answers (request index 0); free with tm_result_free */
    double submit_ms;  /* milliseconds since tm_serve_start: submitted, */
    double start_ms;   /*   its batch admitted, */
    double done_ms;    /*   answers complete */
} tm_completion;

/* config may be null (defaults). TM_ERR_STATE if already serving or the tensor-core
 * kernel is not available. */
int tm_serve_start(tm_ctx *ctx, const tm_serve_config *config);
int tm_submit(tm_ctx *ctx, const tm_request *request, uint64_t *ticket);
/* Up to `capacity` completions; waits up to timeout_ms for the first (0: no wait, <0: no
 * limit). *count = completions written. */
int tm_poll(tm_ctx *ctx, tm_completion *out, int capacity, int timeout_ms, int *count);
/* Completes everything submitted, then stops the workers; completions stay pollable
 * until the next tm_serve_start or tm_ctx_destroy (which stops serving too). */
int tm_serve_stop(tm_ctx *ctx);
/* Requests queued, requests in batches on the GPU, their admitted device bytes, and the
 * kernel launches of the served batches so far (any pointer may be null). */
int tm_serve_status(tm_ctx *ctx, uint64_t *pending, uint64_t *in_flight, uint64_t *in_flight_bytes,
                    uint64_t *launches);

#ifdef __cplusplus
}
#endif

#endif
