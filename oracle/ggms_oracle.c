/* ggms_oracle.c -- CPU sort-and-choose oracle (plain C, single thread).
 *
 * TEST INFRASTRUCTURE ONLY (see ggms_oracle.h).  This is the checker the CUDA
 * path is compared against; the product never calls it.
 *
 * Restated from the reference (FrzNo1/GGMS-Distributed, DistributedSMOS/):
 *   timeSortAndChooseMultiselect  iterativeSMOSTimingFunctions.cu:76-120
 *       thrust::sort ascending of the whole vector, then
 *   copyInChunk                   iterativeSMOSTimingFunctions.cu:67-73
 *       out[i] = sorted[numElements - kList[i]]      (k = 1 -> maximum)
 * Sorting is an LSD radix sort (8-bit digits) of the order-preserving keys, so
 * the answer is the bit pattern of the chosen element.
 */
#include "ggms_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ---- order-preserving key maps ------------------------------------------------
 * float: flip all bits of negatives, flip only the sign bit of non-negatives.  */
uint32_t ggms_oracle_key_f32(float v) {
  uint32_t u;
  memcpy(&u, &v, 4);
  return u ^ ((u >> 31) ? 0xFFFFFFFFu : 0x80000000u);
}
uint64_t ggms_oracle_key_f64(double v) {
  uint64_t u;
  memcpy(&u, &v, 8);
  return u ^ ((u >> 63) ? 0xFFFFFFFFFFFFFFFFull : 0x8000000000000000ull);
}
uint32_t ggms_oracle_key_u32(uint32_t v) { return v; }
uint32_t ggms_oracle_key_i32(int32_t v) { return ((uint32_t)v) ^ 0x80000000u; }
float ggms_oracle_unkey_f32(uint32_t k) {
  uint32_t u = k ^ ((k >> 31) ? 0x80000000u : 0xFFFFFFFFu);
  float v;
  memcpy(&v, &u, 4);
  return v;
}
double ggms_oracle_unkey_f64(uint64_t k) {
  uint64_t u = k ^ ((k >> 63) ? 0x8000000000000000ull : 0xFFFFFFFFFFFFFFFFull);
  double v;
  memcpy(&v, &u, 8);
  return v;
}

/* ---- LSD radix sorts ----------------------------------------------------------- */
static void radix_sort_u32(uint32_t* a, uint32_t* tmp, int64_t n) {
  for (int shift = 0; shift < 32; shift += 8) {
    int64_t cnt[257];
    memset(cnt, 0, sizeof cnt);
    for (int64_t i = 0; i < n; ++i) cnt[((a[i] >> shift) & 0xFF) + 1]++;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (int64_t i = 0; i < n; ++i) tmp[cnt[(a[i] >> shift) & 0xFF]++] = a[i];
    uint32_t* t = a; a = tmp; tmp = t;
  }
  /* 4 passes: the sorted data is back in the caller's first buffer */
}
static void radix_sort_u64(uint64_t* a, uint64_t* tmp, int64_t n) {
  for (int shift = 0; shift < 64; shift += 8) {
    int64_t cnt[257];
    memset(cnt, 0, sizeof cnt);
    for (int64_t i = 0; i < n; ++i) cnt[((a[i] >> shift) & 0xFF) + 1]++;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (int64_t i = 0; i < n; ++i) tmp[cnt[(a[i] >> shift) & 0xFF]++] = a[i];
    uint64_t* t = a; a = tmp; tmp = t;
  }
  /* 8 passes: the sorted data is back in the caller's first buffer */
}

static int ks_ok(int64_t n, const uint32_t* ks, int64_t nk) {
  if (n <= 0 || nk < 0 || (nk > 0 && !ks)) return 0;
  for (int64_t i = 0; i < nk; ++i)
    if (ks[i] < 1u || (int64_t)ks[i] > n) return 0;
  return 1;
}

/* sort-and-choose on 32-bit keys; keys[] is overwritten with the sorted keys */
static int choose32(uint32_t* keys, int64_t n, const uint32_t* ks, int64_t nk, uint32_t* out_keys) {
  uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
  if (!tmp) return -1;
  radix_sort_u32(keys, tmp, n);
  free(tmp);
  for (int64_t i = 0; i < nk; ++i) out_keys[i] = keys[n - (int64_t)ks[i]];
  return 0;
}

#define SELECT32(SUF, T, TOKEY, FROMKEY)                                                  \
  int ggms_oracle_select_##SUF(const T* in, int64_t n, const uint32_t* ks, int64_t nk,   \
                               T* out) {                                                  \
    if (!in || !out || !ks_ok(n, ks, nk)) return -1;                                      \
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);                     \
    uint32_t* ok = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(nk > 0 ? nk : 1));       \
    if (!keys || !ok) { free(keys); free(ok); return -1; }                                 \
    for (int64_t i = 0; i < n; ++i) keys[i] = TOKEY(in[i]);                               \
    int rc = choose32(keys, n, ks, nk, ok);                                               \
    if (rc == 0)                                                                          \
      for (int64_t i = 0; i < nk; ++i) out[i] = FROMKEY(ok[i]);                            \
    free(keys);                                                                           \
    free(ok);                                                                             \
    return rc;                                                                            \
  }

static uint32_t unkey_u32(uint32_t k) { return k; }
static int32_t unkey_i32(uint32_t k) { return (int32_t)(k ^ 0x80000000u); }

SELECT32(f32, float, ggms_oracle_key_f32, ggms_oracle_unkey_f32)
SELECT32(u32, uint32_t, ggms_oracle_key_u32, unkey_u32)
SELECT32(i32, int32_t, ggms_oracle_key_i32, unkey_i32)

int ggms_oracle_select_f64(const double* in, int64_t n, const uint32_t* ks, int64_t nk,
                           double* out) {
  if (!in || !out || !ks_ok(n, ks, nk)) return -1;
  uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  if (!keys || !tmp) { free(keys); free(tmp); return -1; }
  for (int64_t i = 0; i < n; ++i) keys[i] = ggms_oracle_key_f64(in[i]);
  radix_sort_u64(keys, tmp, n);
  for (int64_t i = 0; i < nk; ++i) out[i] = ggms_oracle_unkey_f64(keys[n - (int64_t)ks[i]]);
  free(keys);
  free(tmp);
  return 0;
}

/* ---- segmented ------------------------------------------------------------------ */
int ggms_oracle_select_segmented_f32(const float* in, const int64_t* seg_off, int64_t nseg,
                                     const uint32_t* ks, const int64_t* k_off, float* out) {
  if (!in || !seg_off || !k_off || nseg < 0) return -1;
  for (int64_t s = 0; s < nseg; ++s) {
    int64_t len = seg_off[s + 1] - seg_off[s];
    int64_t nk = k_off[s + 1] - k_off[s];
    if (nk == 0) continue;
    if (ggms_oracle_select_f32(in + seg_off[s], len, ks + k_off[s], nk, out + k_off[s]) != 0)
      return -1;
  }
  return 0;
}
int ggms_oracle_select_segmented_u32(const uint32_t* in, const int64_t* seg_off, int64_t nseg,
                                     const uint32_t* ks, const int64_t* k_off, uint32_t* out) {
  if (!in || !seg_off || !k_off || nseg < 0) return -1;
  for (int64_t s = 0; s < nseg; ++s) {
    int64_t len = seg_off[s + 1] - seg_off[s];
    int64_t nk = k_off[s + 1] - k_off[s];
    if (nk == 0) continue;
    if (ggms_oracle_select_u32(in + seg_off[s], len, ks + k_off[s], nk, out + k_off[s]) != 0)
      return -1;
  }
  return 0;
}
