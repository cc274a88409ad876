// ggms_compat.hpp -- the reference's C++ entry points, header-only, over the C ABI.
//
// A caller of FrzNo1/GGMS-Distributed's single-GPU path includes this header
// instead of bucketMultiselect.cuh / iterativeSMOS.cuh and links
// libggms_b200.so; the call sites stay as they are:
//
//   BucketMultiselect::bucketMultiselectWrapper(d_vec, n, kVals, kCount, out,
//                                               dp.multiProcessorCount,
//                                               dp.maxThreadsPerBlock);
//   IterativeSMOS::iterativeSMOSWrapper(...same arguments...);
//
// Reference declarations replaced:
//   DistributedSMOS/bucketMultiselect.cuh:101-107  (template, namespace BucketMultiselect)
//   DistributedSMOS/iterativeSMOS.cuh:214-220      (template, namespace IterativeSMOS)
// instantiated for int, unsigned int, float and double like the reference
// (bucketMultiselect.cu:888-899, iterativeSMOS.cu:1604-1612).
//
// Behaviour kept: k is the 1-based k-th largest; d_vector is device memory;
// kVals and outputs are host memory; the return value is (T)1 as in the
// reference (bucketMultiselect.cu:885, iterativeSMOS.cu:1601); on an error a
// line "Error at <file>:<line>" is printed like the reference's CUDA_CALL
// macro (bucketMultiselect.cu:35-37) -- here with the status text.
// Behaviour changed: the answers are exact in every case (the reference's
// iterativeSMOS can return an arbitrary element of a stalled bucket,
// iterativeSMOS.cu:1515-1531), and d_vector is never modified (the reference's
// iterativeSMOS compacts into it, iterativeSMOS.cu:1370-1377).
// ggms_last_status() returns the status of the last call on this thread.
#pragma once
#include <cstdio>

#include "ggms.h"

namespace ggms_compat_detail {
inline int& last_status() {
  static thread_local int s = GGMS_OK;
  return s;
}
inline void report(int s, const char* file, int line) {
  last_status() = s;
  if (s != GGMS_OK) printf("Error at %s:%d (%s)\n", file, line, ggms_status_string(s));
}
inline int bucket(float* d, int n, unsigned* k, int nk, float* o, int b, int t) {
  return ggms_bucket_multiselect_f32(d, n, k, nk, o, b, t);
}
inline int bucket(double* d, int n, unsigned* k, int nk, double* o, int b, int t) {
  return ggms_bucket_multiselect_f64(d, n, k, nk, o, b, t);
}
inline int bucket(unsigned* d, int n, unsigned* k, int nk, unsigned* o, int b, int t) {
  return ggms_bucket_multiselect_u32(d, n, k, nk, o, b, t);
}
inline int bucket(int* d, int n, unsigned* k, int nk, int* o, int b, int t) {
  return ggms_bucket_multiselect_i32(d, n, k, nk, o, b, t);
}
inline int iterative(float* d, int n, unsigned* k, int nk, float* o, int b, int t) {
  return ggms_iterative_smos_f32(d, n, k, nk, o, b, t);
}
inline int iterative(double* d, int n, unsigned* k, int nk, double* o, int b, int t) {
  return ggms_iterative_smos_f64(d, n, k, nk, o, b, t);
}
inline int iterative(unsigned* d, int n, unsigned* k, int nk, unsigned* o, int b, int t) {
  return ggms_iterative_smos_u32(d, n, k, nk, o, b, t);
}
inline int iterative(int* d, int n, unsigned* k, int nk, int* o, int b, int t) {
  return ggms_iterative_smos_i32(d, n, k, nk, o, b, t);
}
}  // namespace ggms_compat_detail

inline int ggms_last_status() { return ggms_compat_detail::last_status(); }

namespace BucketMultiselect {
template <typename T>
T bucketMultiselectWrapper(T* d_vector, int length, unsigned int* kVals_ori, int numKs,
                           T* outputs, int blocks, int threads) {
  int s = ggms_compat_detail::bucket(d_vector, length, kVals_ori, numKs, outputs, blocks, threads);
  ggms_compat_detail::report(s, __FILE__, __LINE__);
  return (T)1;
}
}  // namespace BucketMultiselect

namespace IterativeSMOS {
template <typename T>
T iterativeSMOSWrapper(T* d_vector, int length, unsigned int* kVals_ori, int numKs, T* outputs,
                       int blocks, int threads) {
  int s = ggms_compat_detail::iterative(d_vector, length, kVals_ori, numKs, outputs, blocks, threads);
  ggms_compat_detail::report(s, __FILE__, __LINE__);
  return (T)1;
}
}  // namespace IterativeSMOS
