/* ggms.h -- C ABI of the B200-native multiple-order-statistic selector.
 *
 * Selects many order statistics (k-th largest values, k 1-based) from a vector
 * that already lives in GPU memory.  Every answer is exact: values are mapped
 * to order-preserving integer keys, so the result is the bit pattern that a
 * sort-and-choose of the same vector would return, duplicates, signed zeros
 * and NaNs included (order: -NaN < -Inf < ... < -0.0 < +0.0 < ... < +Inf < +NaN).
 *
 * Plain C: pointers, sizes and status codes only.  The CUDA stream is passed as
 * `void*` (a cudaStream_t); NULL means the legacy default stream.
 *
 * Reference interfaces replaced (FrzNo1/GGMS-Distributed, DistributedSMOS/):
 *   BucketMultiselect::bucketMultiselectWrapper<T>  bucketMultiselect.cuh:101-107
 *                                                    (definition bucketMultiselect.cu:853-886)
 *   IterativeSMOS::iterativeSMOSWrapper<T>          iterativeSMOS.cuh:214-220
 *                                                    (definition iterativeSMOS.cu:1580-1602)
 * Both are instantiated there for int, unsigned int, float and double
 * (bucketMultiselect.cu:888-899, iterativeSMOS.cu:1604-1612); the _i32, _u32,
 * _f32 and _f64 entry points below are those four instantiations.
 * The header-only C++ shims with the reference's exact names are in
 * ggms_compat.hpp.
 */
#ifndef GGMS_H
#define GGMS_H

#include <stdint.h>

#if defined(__GNUC__)
#define GGMS_API __attribute__((visibility("default")))
#else
#define GGMS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference returns a constant 1 and prints on error;
 *      these entry points return one of these instead) ---- */
enum {
  GGMS_OK = 0,
  GGMS_E_INVALID_ARG = 1,   /* null pointer, length <= 0, numKs < 0, k outside [1, length] */
  GGMS_E_OOM = 2,           /* device or pinned host allocation failed */
  GGMS_E_NOT_CONVERGED = 3, /* a k was not resolved within the level limit (never expected) */
  GGMS_E_CUDA = 4,          /* a CUDA runtime call failed */
  GGMS_E_UNSUPPORTED = 5,   /* option combination not supported */
  GGMS_E_INTERNAL = 6       /* internal consistency check failed (device error word) */
};

/* ---- level-0 bucket assigners ---- */
enum {
  GGMS_ASSIGNER_AUTO = 0,        /* learned PL-CDF, sampled pivots if its imbalance is over the bound */
  GGMS_ASSIGNER_SAMPLED = 1,     /* sampled pivots + per-segment slopes (the reference's method) */
  GGMS_ASSIGNER_LEARNED_PL = 2,  /* monotone piecewise-linear CDF, trained on the GPU */
  GGMS_ASSIGNER_LEARNED_MLP = 3  /* monotone 1-32-32-1 MLP CDF, trained on the GPU */
};

/* Filled on request (opts->stats != NULL); costs one extra stream sync. */
typedef struct ggms_stats {
  int32_t assigner_used;        /* GGMS_ASSIGNER_* that produced the level-0 buckets */
  int32_t num_buckets;          /* level-0 buckets */
  int32_t full_passes;          /* launches that read the whole input, counted by those kernels on the
                                   device: 2 on the single-vector path (PASS 1 and PASS 2); on the
                                   batched path the level-0 count and copy when a segment needs them */
  int32_t levels;               /* refinement levels that ran over candidates */
  int64_t candidates;           /* elements the level-0 compaction copied */
  int64_t refine_elements;      /* elements read by all refinement levels together */
  int32_t active_buckets;       /* level-0 buckets holding at least one requested k */
  int32_t point_buckets;        /* active level-0 buckets holding a single key (no copy needed) */
  int32_t small_segments;       /* segments finished by the in-shared-memory select */
  int32_t sample_size;          /* keys drawn for the assigner */
  float bucket_max_over_mean;   /* level-0 occupancy: max bucket / (n / num_buckets) */
  float model_imbalance;        /* max/mean of the model's buckets on its own sample (learned) */
  float model_loss;             /* final training loss of the learned model (PL: squared CDF error over
                                   its sample; MLP: mean squared logit error at its training points) */
  int32_t window_runs;          /* PASS 1 windows: bucket runs PASS 1 bucketed (0: every key bucketed) */
  int32_t model_segments;       /* segments of the learned model's piecewise-linear form (0: sampled);
                                   written only for callers whose opts carry pl_knots */
} ggms_stats;

typedef struct ggms_opts {
  int32_t struct_size;          /* sizeof(ggms_opts) */
  int32_t assigner;             /* GGMS_ASSIGNER_* */
  int32_t num_buckets;          /* level-0 buckets: power of two in [2^10, 2^15]; 0 = auto */
  int32_t sample_size;          /* keys sampled for the assigner: power of two in [2^10, 2^16]; 0 = auto */
  uint64_t seed;                /* sample positions are a hash of (seed, i) */
  float imbalance_bound;        /* learned model -> sampled fallback above this max/mean; 0 = 3.0 */
  int32_t train_steps;          /* optimizer steps for the learned models; 0 = auto */
  int32_t ks_on_device;         /* 1: the k array is device memory */
  int32_t out_on_device;        /* 1: the output array is device memory */
  int32_t pass_threads;         /* CTA size of the two passes: 256, 512 or 1024; 0 = tuned default */
  int32_t pass_unroll;          /* how the passes stream the input: 2, 4 or 8 16-byte loads in flight
                                   per thread (registers); -1 = 32 KB chunks staged by bulk copies (TMA)
                                   in a ring of shared-memory stages; -2 = 16 KB chunks copied by every
                                   thread with cp.async into its own shared-memory slots, three chunks
                                   ahead (-1 and -2: pass_threads 1024 only); 0 = the default (4) */
  float window_z;               /* PASS 1 windows: safety margin of the predicted k positions in
                                   binomial standard deviations; 0 = 6; < 0 = no windows */
  int32_t autotune;             /* 1: when num_buckets and the pass shape are left at 0, the first call of a
                                   shape class times the candidates on the caller's data and the context
                                   keeps the fastest (the batched path tunes its level kernels' CTAs) */
  ggms_stats* stats;            /* optional host pointer */
  int32_t pl_knots;             /* segments of the learned piecewise-linear CDF model: 16..1024;
                                   0 = auto (PL: min(512, num_buckets / 4); MLP: min(1024,
                                   num_buckets / 4)).  Appended last: a caller
                                   built against the layout without it (struct_size = its offset)
                                   is still accepted and gets the default */
  int32_t pad0;
} ggms_opts;

GGMS_API void ggms_default_opts(ggms_opts* opts);
GGMS_API const char* ggms_status_string(int status);
GGMS_API int ggms_version(void);

/* A context owns a device workspace (grown on demand and reused), pinned
 * staging buffers and events.  One context must not be used by two host threads
 * at once; distinct contexts are independent. */
typedef struct ggms_context ggms_context;
GGMS_API int ggms_create(ggms_context** ctx, int device);
GGMS_API int ggms_destroy(ggms_context* ctx);
/* The context the drop-in entry points use on the current device. */
GGMS_API int ggms_get_default_context(ggms_context** ctx);

/* Profiling hooks (no reference counterpart; the reference's own timer is a
 * printf around commented-out calls, DistributedSMOS/bucketMultiselect.cu:54-72).
 * While enabled, every single-vector call records CUDA events on its own
 * stream around PASS 1 (l0_count) and PASS 2 (l0_compact) and around the whole
 * call; no host sync is added.  ggms_context_pass_times drains up to `max`
 * recorded calls (oldest first, waiting for their events) into the three
 * arrays and returns how many it wrote.  ggms_context_launches counts every
 * kernel this context has launched. */
GGMS_API int ggms_context_profile(ggms_context* ctx, int enable);
GGMS_API int ggms_context_pass_times(ggms_context* ctx, float* pass1_ms, float* pass2_ms,
                                     float* call_ms, int max);
/* Per-phase device times of profiled single-vector calls (drains the same ring
 * as ggms_context_pass_times): for each call GGMS_PHASES floats, in order
 *   0 k set-up, sample and sample sort   1 assigner (sampled and learned)
 *   2 PASS 1 windows                     3 PASS 1 (count)
 *   4 between the passes (scan, locate, children, write cursors)
 *   5 PASS 2 (copy)                      6 finishing (in-shared-memory select,
 *                                          refinement levels)
 *   7 answers (write-out, copies)
 * Returns the number of calls written (at most `max`), or -status. */
#define GGMS_PHASES 8
GGMS_API int ggms_context_phase_times(ggms_context* ctx, float* ms, int max);

/* Device-side status of the last call this context enqueued (no reference
 * counterpart: the reference is synchronous and prints).  Calls whose ks and
 * answers both live in device memory return GGMS_OK without a host sync, so a
 * problem only the device can see -- a device-resident k outside [1, n], a
 * decreasing segment offset, a failed internal check -- is recorded in the
 * call's device counters instead.  This waits for that call (and, if `stream`
 * is not NULL, for the work enqueued on `stream` before it) and stores its
 * GGMS_* status in *status.  Host-synchronous calls already return it.  The
 * next call of the context overwrites it. */
GGMS_API int ggms_context_status(ggms_context* ctx, void* stream, int* status);
GGMS_API int64_t ggms_context_launches(ggms_context* ctx);
/* Calls of this context that ran as a replay of a captured CUDA graph: a call
 * whose arguments, options and workspace repeat is captured the second time
 * it is seen (on a private stream) and replayed from then on; statistics and
 * profiling calls always run directly. */
GGMS_API int64_t ggms_context_graph_launches(ggms_context* ctx);

/* ---- drop-in entry points: the reference's wrapper signatures in C spelling ----
 * d_vector: device memory, `length` elements, never modified (the reference's
 *           iterativeSMOS may overwrite it; this one never does).
 * kVals:    host memory, numKs entries, 1-based k-th LARGEST, read only.
 * outputs:  host memory, numKs entries, answers in the caller's k order.
 * blocks, threads: launch-geometry hints of the reference (multiProcessorCount,
 *           maxThreadsPerBlock); accepted and ignored -- the launch shapes are
 *           chosen by the library.
 * Synchronous: returns after the outputs are in host memory.  Uses a
 * per-device default context guarded by a mutex and the legacy default stream. */
GGMS_API int ggms_bucket_multiselect_f32(const float* d_vector, int length, const uint32_t* kVals,
                                int numKs, float* outputs, int blocks, int threads);
GGMS_API int ggms_bucket_multiselect_f64(const double* d_vector, int length, const uint32_t* kVals,
                                int numKs, double* outputs, int blocks, int threads);
GGMS_API int ggms_bucket_multiselect_u32(const uint32_t* d_vector, int length, const uint32_t* kVals,
                                int numKs, uint32_t* outputs, int blocks, int threads);
GGMS_API int ggms_bucket_multiselect_i32(const int32_t* d_vector, int length, const uint32_t* kVals,
                                int numKs, int32_t* outputs, int blocks, int threads);

GGMS_API int ggms_iterative_smos_f32(const float* d_vector, int length, const uint32_t* kVals,
                            int numKs, float* outputs, int blocks, int threads);
GGMS_API int ggms_iterative_smos_f64(const double* d_vector, int length, const uint32_t* kVals,
                            int numKs, double* outputs, int blocks, int threads);
GGMS_API int ggms_iterative_smos_u32(const uint32_t* d_vector, int length, const uint32_t* kVals,
                            int numKs, uint32_t* outputs, int blocks, int threads);
GGMS_API int ggms_iterative_smos_i32(const int32_t* d_vector, int length, const uint32_t* kVals,
                            int numKs, int32_t* outputs, int blocks, int threads);

/* ---- extended single-vector entry points ----
 * Same semantics; the k and output arrays may be host or device memory
 * (opts->ks_on_device / out_on_device), work is enqueued on `stream`.
 * With both arrays on the device the call is asynchronous (no host sync)
 * unless opts->stats is set; a device-resident k outside [1, n] is then
 * reported by ggms_context_status, not by the return value.  1 <= n <= 2^32 - 1. */
GGMS_API int ggms_multiselect_f32_ex(ggms_context* ctx, const float* d_in, int64_t n,
                            const uint32_t* ks, int64_t nk, float* out,
                            const ggms_opts* opts, void* stream);
GGMS_API int ggms_multiselect_f64_ex(ggms_context* ctx, const double* d_in, int64_t n,
                            const uint32_t* ks, int64_t nk, double* out,
                            const ggms_opts* opts, void* stream);
GGMS_API int ggms_multiselect_u32_ex(ggms_context* ctx, const uint32_t* d_in, int64_t n,
                            const uint32_t* ks, int64_t nk, uint32_t* out,
                            const ggms_opts* opts, void* stream);
GGMS_API int ggms_multiselect_i32_ex(ggms_context* ctx, const int32_t* d_in, int64_t n,
                            const uint32_t* ks, int64_t nk, int32_t* out,
                            const ggms_opts* opts, void* stream);

/* ---- top-k: the K largest values, largest first ----
 * The reference's timeBucketTopkselect (DistributedSMOS/iterativeSMOSTimingFunctions.cu:307-333)
 * runs bucketMultiselect with ks = 1..K; this does the same on the device (no
 * k array is uploaded): out[i] = the (i+1)-th largest, exact.  `out` is host
 * memory unless opts->out_on_device.  1 <= K <= n. */
GGMS_API int ggms_topk_f32(ggms_context* ctx, const float* d_in, int64_t n, int64_t K, float* out,
                           const ggms_opts* opts, void* stream);
GGMS_API int ggms_topk_f64(ggms_context* ctx, const double* d_in, int64_t n, int64_t K, double* out,
                           const ggms_opts* opts, void* stream);
GGMS_API int ggms_topk_u32(ggms_context* ctx, const uint32_t* d_in, int64_t n, int64_t K, uint32_t* out,
                           const ggms_opts* opts, void* stream);
GGMS_API int ggms_topk_i32(ggms_context* ctx, const int32_t* d_in, int64_t n, int64_t K, int32_t* out,
                           const ggms_opts* opts, void* stream);

/* ---- batched segmented selection (no reference counterpart: the reference has
 *      no batched API; its callers loop over per-vector wrapper calls) ----
 * Segment s is d_in[seg_off[s] .. seg_off[s+1]); its ks are
 * ks[k_off[s] .. k_off[s+1]) (1-based k-th largest within the segment) and its
 * answers go to out[k_off[s] .. k_off[s+1]).  seg_off and k_off hold nseg+1
 * entries; all five arrays are DEVICE memory.  Work is enqueued on `stream`,
 * but the call first reads seg_off[0], seg_off[nseg], k_off[0] and k_off[nseg]
 * back to the host (the totals size the workspace): one host sync on `stream`
 * per call, so the call cannot itself be captured into the caller's CUDA graph
 * (repeated calls replay the library's own graph).  Errors that only the
 * device sees (a k outside its segment, seg_off decreasing) are reported by
 * ggms_context_status. */
GGMS_API int ggms_multiselect_segmented_f32(ggms_context* ctx, const float* d_in, const int64_t* seg_off,
                                   int64_t nseg, const uint32_t* ks, const int64_t* k_off,
                                   float* out, const ggms_opts* opts, void* stream);
GGMS_API int ggms_multiselect_segmented_u32(ggms_context* ctx, const uint32_t* d_in, const int64_t* seg_off,
                                   int64_t nseg, const uint32_t* ks, const int64_t* k_off,
                                   uint32_t* out, const ggms_opts* opts, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GGMS_H */
