// A caller of the reference's C++ entry points, written the way the
// reference's own timing functions call them
// (DistributedSMOS/iterativeSMOSTimingFunctions.cu:134-156 and 207-229:
// unsigned length and count, uint* kVals, host outputs, the device's SM count
// and block size as the launch hints), built against include/ggms_compat.hpp
// and linked to libggms_b200.so instead of the reference's sources.
//
//   caller <type: i32|u32|f32|f64> <entry: bucket|iterative> values.bin ks.bin out.bin
//
// values.bin holds the raw values, ks.bin uint32 ks (1-based k-th largest);
// out.bin receives the answers.  Exit status 0 only when every step and the
// library's own status (ggms_last_status) succeeded.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "ggms_compat.hpp"

typedef unsigned int uint;

template <typename T>
struct results_t {  // the shape of the reference's result holder
  float time;
  T* vals;
};

static std::vector<char> slurp(const char* path) {
  std::vector<char> b;
  FILE* f = std::fopen(path, "rb");
  if (!f) return b;
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  b.resize((size_t)sz);
  if (sz > 0 && std::fread(b.data(), 1, (size_t)sz, f) != (size_t)sz) b.clear();
  std::fclose(f);
  return b;
}

template <typename T>
static int run(bool iterative, const char* vpath, const char* kpath, const char* opath) {
  const std::vector<char> vb = slurp(vpath), kb = slurp(kpath);
  if (vb.empty() || kb.empty() || vb.size() % sizeof(T) || kb.size() % 4) return 2;
  uint numElements = (uint)(vb.size() / sizeof(T));
  uint kCount = (uint)(kb.size() / 4);
  std::vector<uint> kv(kCount);
  std::memcpy(kv.data(), kb.data(), kb.size());
  uint* kVals = kv.data();
  results_t<T> res;
  std::vector<T> out(kCount);
  res.vals = out.data();
  cudaDeviceProp dp;
  if (cudaGetDeviceProperties(&dp, 0) != cudaSuccess) return 3;
  T* d_vec = nullptr;
  if (cudaMalloc(&d_vec, vb.size()) != cudaSuccess) return 3;
  if (cudaMemcpy(d_vec, vb.data(), vb.size(), cudaMemcpyHostToDevice) != cudaSuccess) return 3;
  T one;
  if (iterative)
    one = IterativeSMOS::iterativeSMOSWrapper(d_vec, numElements, kVals, kCount, res.vals,
                                              dp.multiProcessorCount, dp.maxThreadsPerBlock);
  else
    one = BucketMultiselect::bucketMultiselectWrapper(d_vec, numElements, kVals, kCount, res.vals,
                                                      dp.multiProcessorCount, dp.maxThreadsPerBlock);
  cudaFree(d_vec);
  if (one != (T)1 || ggms_last_status() != GGMS_OK) return 4;
  FILE* f = std::fopen(opath, "wb");
  if (!f || std::fwrite(out.data(), sizeof(T), kCount, f) != kCount) return 5;
  std::fclose(f);
  return 0;
}

int main(int argc, char** argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s <i32|u32|f32|f64> <bucket|iterative> values ks out\n", argv[0]);
    return 1;
  }
  const bool it = std::strcmp(argv[2], "iterative") == 0;
  if (!std::strcmp(argv[1], "i32")) return run<int>(it, argv[3], argv[4], argv[5]);
  if (!std::strcmp(argv[1], "u32")) return run<unsigned int>(it, argv[3], argv[4], argv[5]);
  if (!std::strcmp(argv[1], "f32")) return run<float>(it, argv[3], argv[4], argv[5]);
  if (!std::strcmp(argv[1], "f64")) return run<double>(it, argv[3], argv[4], argv[5]);
  return 1;
}
