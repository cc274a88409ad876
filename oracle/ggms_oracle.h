/* ggms_oracle.h -- CPU oracle for exact multiple-order-statistic selection.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load this library, and only as the
 * checker or the timed CPU baseline -- never as the product path.
 *
 * What it restates (reference: FrzNo1/GGMS-Distributed, DistributedSMOS/):
 *   - timeSortAndChooseMultiselect + copyInChunk
 *     (iterativeSMOSTimingFunctions.cu:67-73, 76-120): sort the whole vector
 *     ascending, answer k with sorted[n - k]  (k = 1 is the maximum).
 *   - the k convention of the drop-in wrappers: k is the 1-based k-th LARGEST
 *     (bucketMultiselect.cu:859-861 and iterativeSMOS.cu:1586-1588 turn it into
 *     the (n-k+1)-th smallest before the core runs).
 * The order used is the total order of the order-preserving integer key
 * (ggms_oracle_key_* below), so NaN, -0.0/+0.0 and duplicates have one
 * defined answer:  -NaN < -Inf < ... < -0.0 < +0.0 < ... < +Inf < +NaN.
 * On NaN- and signed-zero-free data this coincides with thrust::sort's order,
 * which is what the reference uses.
 */
#ifndef GGMS_ORACLE_H
#define GGMS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* order-preserving key maps and their inverses */
uint32_t ggms_oracle_key_f32(float v);
uint64_t ggms_oracle_key_f64(double v);
uint32_t ggms_oracle_key_u32(uint32_t v);
uint32_t ggms_oracle_key_i32(int32_t v);
float    ggms_oracle_unkey_f32(uint32_t k);
double   ggms_oracle_unkey_f64(uint64_t k);

/* Sort-and-choose over one vector.  ks are 1-based k-th largest.
 * Returns 0 on success, -1 on a bad argument (n <= 0, k outside [1, n]). */
int ggms_oracle_select_f32(const float*    in, int64_t n, const uint32_t* ks, int64_t nk, float*    out);
int ggms_oracle_select_f64(const double*   in, int64_t n, const uint32_t* ks, int64_t nk, double*   out);
int ggms_oracle_select_u32(const uint32_t* in, int64_t n, const uint32_t* ks, int64_t nk, uint32_t* out);
int ggms_oracle_select_i32(const int32_t*  in, int64_t n, const uint32_t* ks, int64_t nk, int32_t*  out);

/* Segmented: segment s is in[seg_off[s] .. seg_off[s+1]), its ks are
 * ks[k_off[s] .. k_off[s+1]) (k-th largest within the segment); answers go to
 * out[k_off[s] + j]. */
int ggms_oracle_select_segmented_f32(const float* in, const int64_t* seg_off, int64_t nseg,
                                     const uint32_t* ks, const int64_t* k_off, float* out);
int ggms_oracle_select_segmented_u32(const uint32_t* in, const int64_t* seg_off, int64_t nseg,
                                     const uint32_t* ks, const int64_t* k_off, uint32_t* out);

/* Multithreaded CPU baselines (ggms_cpu_baseline.cpp, OpenMP).
 * method 0: parallel sort of the keys, then pick;  method 1: recursive
 * std::nth_element over the sorted k list, split at the median k, OpenMP tasks.
 * threads <= 0 means all hardware threads.  Returns 0 or -1. */
int ggms_cpu_multiselect_f32(const float* in, int64_t n, const uint32_t* ks, int64_t nk,
                             float* out, int threads, int method);
int ggms_cpu_multiselect_f64(const double* in, int64_t n, const uint32_t* ks, int64_t nk,
                             double* out, int threads, int method);
int ggms_cpu_multiselect_u32(const uint32_t* in, int64_t n, const uint32_t* ks, int64_t nk,
                             uint32_t* out, int threads, int method);
/* Segmented (the oracle's segmented layout): each segment by method 1, the
 * segments spread over the threads.  Returns 0 or -1. */
int ggms_cpu_multiselect_segmented_f32(const float* in, const int64_t* seg_off, int64_t nseg,
                                       const uint32_t* ks, const int64_t* k_off, float* out, int threads);
int ggms_cpu_multiselect_segmented_u32(const uint32_t* in, const int64_t* seg_off, int64_t nseg,
                                       const uint32_t* ks, const int64_t* k_off, uint32_t* out, int threads);
int ggms_cpu_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
