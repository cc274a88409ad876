// ref_capi.cu -- a thin extern "C" veneer over the UNMODIFIED reference build.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's own sources (DistributedSMOS/bucketMultiselect.cu and
// DistributedSMOS/iterativeSMOS.cu, read where they lie) by oracle/Makefile
// into oracle/_ref/libggms_ref.so.  It lets the tests, the golden-vector
// script and bench.py's reference arm call the reference's public entry
// points through ctypes.  Nothing in the product links or loads it.
//
// Entry points wrapped (reference signatures):
//   BucketMultiselect::bucketMultiselectWrapper<T>   DistributedSMOS/bucketMultiselect.cuh:101-107
//   IterativeSMOS::iterativeSMOSWrapper<T>           DistributedSMOS/iterativeSMOS.cuh:214-220
// Timing protocol restated from DistributedSMOS/iterativeSMOSTimingFunctions.cu:42-51,134-156:
//   cudaMalloc + H2D of the vector outside the timer, CUDA events around the
//   wrapper call (the reference's internal allocations and copies included).
//
// Two guards are added around the reference, both on the caller side:
//  * the device copy of the vector is allocated with PAD spare elements, each a
//    copy of element 0.  The reference draws its 1024 sample positions as
//    (int)(u * length) with u from thrust::uniform_real_distribution<float>(0,1)
//    (bucketMultiselect.cu:403-412); that float can round to exactly 1.0f, so
//    the gather may read element [length].  The pad keeps that read inside the
//    allocation and inside [min, max].
//  * a k-list whose every entry is 1 or length is rejected: after peeling those
//    the reference indexes its host arrays at [-1] (bucketMultiselect.cu:640-656,
//    731-742).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>
#include <thrust/device_vector.h>
#include <thrust/functional.h>
#include <thrust/random.h>
#include <thrust/sort.h>

#include "bucketMultiselect.cuh"
#include "iterativeSMOS.cuh"

namespace {

constexpr int PAD = 64;

template <typename T>
int k_list_ok(const unsigned* ks, int nk, int n) {
  if (nk <= 0 || n <= 0) return 0;
  int interior = 0;
  for (int i = 0; i < nk; ++i) {
    if (ks[i] < 1u || ks[i] > (unsigned)n) return 0;
    if (ks[i] != 1u && ks[i] != (unsigned)n) interior = 1;
  }
  return interior;
}

// which: 0 = bucketMultiselect, 1 = iterativeSMOS.
// Returns elapsed milliseconds (reference protocol), or a negative value on a
// rejected argument / CUDA error.
template <typename T>
float run_ref(int which, const T* h_vec, int n, const unsigned* ks, int nk, T* h_out) {
  if (!k_list_ok<T>(ks, nk, n)) return -1.0f;
  cudaDeviceProp dp;
  if (cudaGetDeviceProperties(&dp, 0) != cudaSuccess) return -2.0f;
  T* d_vec = nullptr;
  if (cudaMalloc(&d_vec, (size_t)(n + PAD) * sizeof(T)) != cudaSuccess) return -3.0f;
  cudaMemcpy(d_vec, h_vec, (size_t)n * sizeof(T), cudaMemcpyHostToDevice);
  for (int i = 0; i < PAD; ++i)
    cudaMemcpy(d_vec + n + i, h_vec, sizeof(T), cudaMemcpyHostToDevice);
  // the wrappers take a non-const k pointer; they copy it before use.
  unsigned* kcopy = (unsigned*)malloc(sizeof(unsigned) * (size_t)nk);
  memcpy(kcopy, ks, sizeof(unsigned) * (size_t)nk);
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  cudaDeviceSynchronize();
  cudaEventRecord(start, 0);
  if (which == 0)
    BucketMultiselect::bucketMultiselectWrapper(d_vec, n, kcopy, nk, h_out,
                                                dp.multiProcessorCount, dp.maxThreadsPerBlock);
  else
    IterativeSMOS::iterativeSMOSWrapper(d_vec, n, kcopy, nk, h_out,
                                        dp.multiProcessorCount, dp.maxThreadsPerBlock);
  cudaEventRecord(stop, 0);
  cudaEventSynchronize(stop);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, start, stop);
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  free(kcopy);
  cudaFree(d_vec);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "reference run: %s\n", cudaGetErrorString(e));
    return -4.0f;
  }
  return ms;
}

}  // namespace

#define GGMS_REF_EXPORT(SUF, T)                                                          \
  extern "C" float ggms_ref_bucket_multiselect_##SUF(const T* h_vec, int n,             \
                                                      const unsigned* ks, int nk, T* out) { \
    return run_ref<T>(0, h_vec, n, ks, nk, out);                                         \
  }                                                                                      \
  extern "C" float ggms_ref_iterative_smos_##SUF(const T* h_vec, int n,                 \
                                                  const unsigned* ks, int nk, T* out) {  \
    return run_ref<T>(1, h_vec, n, ks, nk, out);                                         \
  }

GGMS_REF_EXPORT(f32, float)
GGMS_REF_EXPORT(f64, double)
GGMS_REF_EXPORT(u32, unsigned int)
GGMS_REF_EXPORT(i32, int)

extern "C" int ggms_ref_available(void) { return 1; }
