// ggms_cpu_baseline.cpp -- multithreaded CPU multiselect (OpenMP).
//
// TEST INFRASTRUCTURE / REPORTED BASELINE ONLY.  bench.py times this on the
// host cores as the "cpu_baseline"; the tests use it as a fast second checker
// at full sizes.  It is never the product path.
//
// Same semantics as the sort-and-choose oracle (ggms_oracle.c, which restates
// DistributedSMOS/iterativeSMOSTimingFunctions.cu:67-120): k is the 1-based
// k-th largest, the order is that of the order-preserving integer key.
//   method 0: __gnu_parallel::sort of all keys, then sorted[n - k].
//   method 1: multi-select by recursive std::nth_element: sort the distinct
//             target positions, nth_element at the median target, recurse on
//             both halves as OpenMP tasks (O(n log K) work).
#include <omp.h>
#include <parallel/algorithm>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "ggms_oracle.h"

namespace {

template <typename K>
void multi_nth(K* a, int64_t lo, int64_t hi, const int64_t* pos, int64_t plo, int64_t phi) {
  // positions pos[plo..phi) are all in [lo, hi); after return a[p] holds the
  // p-th smallest key of the original range for each such p.
  if (plo >= phi || hi - lo <= 1) return;
  int64_t pm = plo + (phi - plo) / 2;
  int64_t p = pos[pm];
  std::nth_element(a + lo, a + p, a + hi);
  int64_t left_hi = pm, right_lo = pm + 1;
  while (left_hi > plo && pos[left_hi - 1] == p) --left_hi;
  while (right_lo < phi && pos[right_lo] == p) ++right_lo;
  if (hi - lo > (1 << 16)) {
#pragma omp task
    multi_nth(a, lo, p, pos, plo, left_hi);
#pragma omp task
    multi_nth(a, p + 1, hi, pos, right_lo, phi);
#pragma omp taskwait
  } else {
    multi_nth(a, lo, p, pos, plo, left_hi);
    multi_nth(a, p + 1, hi, pos, right_lo, phi);
  }
}

// The same recursion without tasks (one thread per segment in the segmented variant).
template <typename K>
void multi_nth_serial(K* a, int64_t lo, int64_t hi, const int64_t* pos, int64_t plo, int64_t phi) {
  if (plo >= phi || hi - lo <= 1) return;
  int64_t pm = plo + (phi - plo) / 2;
  int64_t p = pos[pm];
  std::nth_element(a + lo, a + p, a + hi);
  int64_t left_hi = pm, right_lo = pm + 1;
  while (left_hi > plo && pos[left_hi - 1] == p) --left_hi;
  while (right_lo < phi && pos[right_lo] == p) ++right_lo;
  multi_nth_serial(a, lo, p, pos, plo, left_hi);
  multi_nth_serial(a, p + 1, hi, pos, right_lo, phi);
}

template <typename K, typename T, typename ToKey, typename FromKey>
int cpu_select(const T* in, int64_t n, const uint32_t* ks, int64_t nk, T* out, int threads,
               int method, ToKey tokey, FromKey fromkey) {
  if (!in || !out || n <= 0 || nk < 0 || (nk > 0 && !ks)) return -1;
  for (int64_t i = 0; i < nk; ++i)
    if (ks[i] < 1u || (int64_t)ks[i] > n) return -1;
  if (threads <= 0) threads = omp_get_max_threads();
  std::vector<K> keys((size_t)n);
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int64_t i = 0; i < n; ++i) keys[(size_t)i] = tokey(in[i]);
  if (method == 0) {
    __gnu_parallel::sort(keys.begin(), keys.end(), std::less<K>(),
                         __gnu_parallel::default_parallel_tag(threads));
  } else {
    std::vector<int64_t> pos((size_t)nk);
    for (int64_t i = 0; i < nk; ++i) pos[(size_t)i] = n - (int64_t)ks[i];
    std::sort(pos.begin(), pos.end());
    pos.erase(std::unique(pos.begin(), pos.end()), pos.end());
#pragma omp parallel num_threads(threads)
#pragma omp single
    multi_nth(keys.data(), 0, n, pos.data(), 0, (int64_t)pos.size());
  }
  for (int64_t i = 0; i < nk; ++i) out[i] = fromkey(keys[(size_t)(n - (int64_t)ks[i])]);
  return 0;
}

// Segmented: every segment by the method-1 multi-select, the segments spread
// over the threads (largest first, dynamic schedule).  Same layout as the
// oracle's ggms_oracle_select_segmented_*.
template <typename K, typename T, typename ToKey, typename FromKey>
int cpu_select_segmented(const T* in, const int64_t* seg_off, int64_t nseg, const uint32_t* ks,
                         const int64_t* k_off, T* out, int threads, ToKey tokey, FromKey fromkey) {
  if (!in || !seg_off || !k_off || !out || nseg <= 0 || seg_off[0] != 0 || k_off[0] != 0) return -1;
  for (int64_t s = 0; s < nseg; ++s) {
    const int64_t len = seg_off[s + 1] - seg_off[s];
    if (len < 0 || k_off[s + 1] < k_off[s]) return -1;
    for (int64_t j = k_off[s]; j < k_off[s + 1]; ++j)
      if (ks[j] < 1u || (int64_t)ks[j] > len) return -1;
  }
  if (threads <= 0) threads = omp_get_max_threads();
  std::vector<int64_t> order((size_t)nseg);
  for (int64_t s = 0; s < nseg; ++s) order[(size_t)s] = s;
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    return seg_off[a + 1] - seg_off[a] > seg_off[b + 1] - seg_off[b];
  });
#pragma omp parallel num_threads(threads)
  {
    std::vector<K> keys;
    std::vector<int64_t> pos;
#pragma omp for schedule(dynamic, 1)
    for (int64_t i = 0; i < nseg; ++i) {
      const int64_t s = order[(size_t)i];
      const int64_t a = seg_off[s], n = seg_off[s + 1] - a, k0 = k_off[s], nk = k_off[s + 1] - k0;
      if (nk == 0) continue;
      keys.resize((size_t)n);
      for (int64_t j = 0; j < n; ++j) keys[(size_t)j] = tokey(in[a + j]);
      pos.resize((size_t)nk);
      for (int64_t j = 0; j < nk; ++j) pos[(size_t)j] = n - (int64_t)ks[k0 + j];
      std::sort(pos.begin(), pos.end());
      pos.erase(std::unique(pos.begin(), pos.end()), pos.end());
      multi_nth_serial(keys.data(), 0, n, pos.data(), 0, (int64_t)pos.size());
      for (int64_t j = 0; j < nk; ++j) out[k0 + j] = fromkey(keys[(size_t)(n - (int64_t)ks[k0 + j])]);
    }
  }
  return 0;
}

}  // namespace

extern "C" int ggms_cpu_max_threads(void) { return omp_get_max_threads(); }

extern "C" int ggms_cpu_multiselect_segmented_f32(const float* in, const int64_t* seg_off, int64_t nseg,
                                                  const uint32_t* ks, const int64_t* k_off, float* out,
                                                  int threads) {
  return cpu_select_segmented<uint32_t>(in, seg_off, nseg, ks, k_off, out, threads, ggms_oracle_key_f32,
                                        ggms_oracle_unkey_f32);
}
extern "C" int ggms_cpu_multiselect_segmented_u32(const uint32_t* in, const int64_t* seg_off, int64_t nseg,
                                                  const uint32_t* ks, const int64_t* k_off, uint32_t* out,
                                                  int threads) {
  return cpu_select_segmented<uint32_t>(in, seg_off, nseg, ks, k_off, out, threads,
                                        [](uint32_t v) { return v; }, [](uint32_t k) { return k; });
}

extern "C" int ggms_cpu_multiselect_f32(const float* in, int64_t n, const uint32_t* ks,
                                        int64_t nk, float* out, int threads, int method) {
  return cpu_select<uint32_t>(in, n, ks, nk, out, threads, method, ggms_oracle_key_f32,
                              ggms_oracle_unkey_f32);
}
extern "C" int ggms_cpu_multiselect_f64(const double* in, int64_t n, const uint32_t* ks,
                                        int64_t nk, double* out, int threads, int method) {
  return cpu_select<uint64_t>(in, n, ks, nk, out, threads, method, ggms_oracle_key_f64,
                              ggms_oracle_unkey_f64);
}
extern "C" int ggms_cpu_multiselect_u32(const uint32_t* in, int64_t n, const uint32_t* ks,
                                        int64_t nk, uint32_t* out, int threads, int method) {
  return cpu_select<uint32_t>(in, n, ks, nk, out, threads, method,
                              [](uint32_t v) { return v; }, [](uint32_t k) { return k; });
}
