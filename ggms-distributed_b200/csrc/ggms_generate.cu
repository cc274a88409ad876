// ggms_generate.cu -- device-side problem generators (include/ggms_generate.h).
//
// One grid-stride kernel per value type; `kind` is uniform across the launch, so the
// switch costs nothing per element.  Every element draws its bits from the SplitMix64
// output function (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014) applied to key + (i + 1) * golden: counter-based, so the
// vector depends only on (kind, n, seed).  Normals use the Box-Muller transform;
// the logarithm, square root, cospi and tan are CUDA's math functions.  The kernels
// only write (4 or 8 bytes per element, coalesced): HBM-write bound.
//
// The reference's tables (DistributedSMOS/generateProblems.cu:75-79, 438-446,
// 509-513) give the kind numbering.  The two KILLER kinds sort their masked sample
// (DistributedSMOS/generateProblems.cu:422-436, 493-507): that sort is CUB's device
// radix sort over the bits the mask leaves, on the caller's stream, into
// stream-ordered scratch (cudaMallocAsync / cudaFreeAsync).

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ggms_generate.h"

namespace ggms_gen {

constexpr uint64_t GOLDEN = 0x9E3779B97F4A7C15ull;

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Per-launch constants: two independent streams of bits and the affine permutation
// that places the two-valued kinds.
struct Params {
  uint64_t key0, key1;
  uint64_t perm_a, perm_b;  // i -> (a i + b) mod n, gcd(a, n) = 1
  uint64_t n;
  int kind;
};

__device__ __forceinline__ uint64_t draw(uint64_t key, uint64_t i) { return mix64(key + (i + 1) * GOLDEN); }

__device__ __forceinline__ float unit24(uint64_t h) { return (float)(h >> 40) * 0x1p-24f; }

__device__ __forceinline__ float normal_f32(uint64_t h) {
  const float u1 = (float)((h >> 40) + 1) * 0x1p-24f;           // (0, 1]
  const float u2 = (float)((h >> 8) & 0xFFFFFFu) * 0x1p-24f;    // [0, 1)
  return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

__device__ __forceinline__ double normal_f64(uint64_t h0, uint64_t h1) {
  const double u1 = (double)((h0 >> 11) + 1) * 0x1p-53;
  const double u2 = (double)(h1 >> 11) * 0x1p-53;
  return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// position of element i in the two-valued layout: a bijection of [0, n), n <= 2^32
__device__ __forceinline__ uint64_t placed(const Params& p, uint64_t i) {
  return (p.perm_a * i % p.n + p.perm_b) % p.n;
}

__global__ void __launch_bounds__(256) gen_f32(float* __restrict__ out, Params p) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride) {
    const uint64_t h = draw(p.key0, i);
    float v;
    switch (p.kind) {
      case 0: v = unit24(h); break;
      case 1: v = normal_f32(h); break;
      case 3: v = fabsf(normal_f32(h)); break;
      case 4: v = normal_f32(h) * 100.0f; break;
      case 5: v = unit24(h) * 1000000.0f; break;
      case 6: v = (placed(p, i) < p.n / 5 ? 1.0f : 0.0f) + 0.01f * normal_f32(draw(p.key1, i)); break;
      case 7: v = 1.0f; break;
      case 8: v = placed(p, i) < p.n / 2 ? 2.0f : 1.0f; break;
      default: {  // 9: Cauchy(0, 1); u in (0, 1) never reaches the poles
        const float u = ((float)(h >> 40) + 0.5f) * 0x1p-24f;
        v = tanf(3.14159265358979f * (u - 0.5f));
      }
    }
    out[i] = v;
  }
}

__global__ void __launch_bounds__(256) gen_f64(double* __restrict__ out, Params p) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride) {
    const uint64_t h = draw(p.key0, i);
    out[i] = p.kind == 0 ? (double)(h >> 11) * 0x1p-53 : normal_f64(h, draw(p.key1, i));
  }
}

__global__ void __launch_bounds__(256) gen_u32(uint32_t* __restrict__ out, Params p) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride) {
    const uint64_t h = draw(p.key0, i);
    uint32_t v;
    if (p.kind == 0) {
      v = (uint32_t)(h >> 32);
    } else if (p.kind == 1) {
      // floor((i + u) 2^32 / n), u = the top 32 bits of h over 2^32: stratum i of n,
      // non-decreasing in i because the low word never carries into i; < 2^32.
      v = (uint32_t)(((i << 32) | (h >> 32)) / p.n);
    } else {
      v = (uint32_t)(i % 100);
    }
    out[i] = v;
  }
}

// KILLER FLOATS / DOUBLES, step 1: the uniform draw of kind 0 with its exponent
// masked away, as bit patterns (generateBucketKillerFloats masks with 0x80EFFFFF,
// generateBucketKillerDoubles with 0x800FFFFFFFFFFFFF): subnormals and, for floats,
// the lowest normal binade.
__global__ void __launch_bounds__(256) killer_draw_f32(uint32_t* __restrict__ out, Params p) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride)
    out[i] = __float_as_uint(unit24(draw(p.key0, i))) & 0x80EFFFFFu;
}

__global__ void __launch_bounds__(256) killer_draw_f64(unsigned long long* __restrict__ out, Params p) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride)
    out[i] = (unsigned long long)__double_as_longlong((double)(draw(p.key0, i) >> 11) * 0x1p-53) &
             0x800FFFFFFFFFFFFFull;
}

// Step 3: the first slots take the powers of two 2^lo .. 2^(lo + count - 1), built
// from their exponent fields (bias: 127 for float, 1023 for double).
template <typename U, int MANT, int BIAS>
__global__ void __launch_bounds__(256) killer_powers(U* __restrict__ out, int lo, int count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) out[i] = (U)(lo + i + BIAS) << MANT;
}

uint64_t gcd64(uint64_t a, uint64_t b) {
  while (b) {
    const uint64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

Params make_params(int64_t n, int kind, uint64_t seed) {
  Params p;
  p.n = (uint64_t)n;
  p.kind = kind;
  p.key0 = mix64(seed + GOLDEN);
  p.key1 = mix64(seed ^ 0xD1B54A32D192ED03ull);
  p.perm_a = 1;
  p.perm_b = 0;
  if (n >= 2) {
    p.perm_a = 1 + mix64(seed ^ 0x5851F42D4C957F2Dull) % (uint64_t)(n - 1);
    while (gcd64(p.perm_a, (uint64_t)n) != 1) p.perm_a = p.perm_a % (uint64_t)(n - 1) + 1;
    p.perm_b = mix64(seed ^ 0x2545F4914F6CDD1Dull) % (uint64_t)n;
  }
  return p;
}

int launch_status() { return cudaGetLastError() == cudaSuccess ? GGMS_OK : GGMS_E_CUDA; }

constexpr int kThreads = 256;

int grid_for(int64_t n) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (n + kThreads - 1) / kThreads;
  const int64_t cap = (int64_t)sms * 8;  // 8 x 256 threads per SM, grid-stride beyond
  return (int)(want < cap ? want : cap);
}

constexpr int64_t kPermMaxN = (int64_t)1 << 32;

// draw (kernel) -> sort the pattern's low `bits` bits (the others are zero) ->
// powers of two at the front; the scratch holds the draw and CUB's temporaries.
template <typename U, int MANT, int BIAS>
int killer(U* d_out, int64_t n, uint64_t seed, cudaStream_t st, int bits, int lo, int npow) {
  size_t tmp_bytes = 0;
  if (cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, (const U*)nullptr, (U*)nullptr, (int)n, 0, bits,
                                     st) != cudaSuccess)
    return GGMS_E_CUDA;
  const size_t keys_bytes = ((size_t)n * sizeof(U) + 255) & ~(size_t)255;
  void* scratch = nullptr;
  if (cudaMallocAsync(&scratch, keys_bytes + tmp_bytes, st) != cudaSuccess) return GGMS_E_CUDA;
  U* keys = (U*)scratch;
  if constexpr (sizeof(U) == 4)
    killer_draw_f32<<<grid_for(n), kThreads, 0, st>>>(keys, make_params(n, 0, seed));
  else
    killer_draw_f64<<<grid_for(n), kThreads, 0, st>>>(keys, make_params(n, 0, seed));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortKeys((uint8_t*)scratch + keys_bytes, tmp_bytes, keys, d_out, (int)n, 0, bits,
                                       st);
  const int count = n < npow ? (int)n : npow;  // the reference writes all npow slots
  if (e == cudaSuccess) {
    killer_powers<U, MANT, BIAS><<<(count + 255) / 256, 256, 0, st>>>(d_out, lo, count);
    e = cudaGetLastError();
  }
  const cudaError_t f = cudaFreeAsync(scratch, st);
  return e == cudaSuccess && f == cudaSuccess ? GGMS_OK : GGMS_E_CUDA;
}

constexpr int64_t kKillerMaxN = ((int64_t)1 << 31) - 1;  // CUB's item count is an int here

}  // namespace ggms_gen

using namespace ggms_gen;

extern "C" GGMS_API int ggms_generate_f32(float* d_out, int64_t n, int kind, uint64_t seed, void* stream) {
  if (!d_out || n <= 0 || kind < 0 || kind > 9) return GGMS_E_INVALID_ARG;
  if ((kind == 6 || kind == 8) && n > kPermMaxN) return GGMS_E_UNSUPPORTED;
  if (kind == 2) {  // KILLER FLOATS: 2^-126 .. 2^126 in the first 253 slots
    if (n > kKillerMaxN) return GGMS_E_UNSUPPORTED;
    return killer<uint32_t, 23, 127>((uint32_t*)d_out, n, seed, (cudaStream_t)stream, 24, -126, 253);
  }
  gen_f32<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(d_out, make_params(n, kind, seed));
  return launch_status();
}

extern "C" GGMS_API int ggms_generate_f64(double* d_out, int64_t n, int kind, uint64_t seed, void* stream) {
  if (!d_out || n <= 0 || kind < 0 || kind > 2) return GGMS_E_INVALID_ARG;
  if (kind == 2) {  // KILLER DOUBLES: 2^-1022 .. 2^1022 in the first 2045 slots
    if (n > kKillerMaxN) return GGMS_E_UNSUPPORTED;
    return killer<unsigned long long, 52, 1023>((unsigned long long*)d_out, n, seed, (cudaStream_t)stream, 52,
                                                -1022, 2045);
  }
  gen_f64<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(d_out, make_params(n, kind, seed));
  return launch_status();
}

extern "C" GGMS_API int ggms_generate_u32(uint32_t* d_out, int64_t n, int kind, uint64_t seed, void* stream) {
  if (!d_out || n <= 0 || kind < 0 || kind > 2) return GGMS_E_INVALID_ARG;
  if (kind == 1 && n > kPermMaxN) return GGMS_E_UNSUPPORTED;
  gen_u32<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(d_out, make_params(n, kind, seed));
  return launch_status();
}
