// ggms_noalloc.cu -- ggms_multiselect_noalloc_f32: exact multiselect that
// allocates nothing.
//
// No counterpart in the reference (its wrappers cudaMalloc/cudaFree inside
// every call, DistributedSMOS/bucketMultiselect.cu:583-606, 805-845).  It is a
// variant of the library's radix refinement levels (count -> locate -> next
// level) that keeps every byte of its state in one file-scope device array:
//
//   scratch (GGMS_NOALLOC_SCRATCH_BYTES, 256-byte aligned, one per device)
//     hist[MAX_KS][256]  per active key prefix, counts of the next 8-bit digit
//     kr[MAX_KS]         per k: its ascending rank inside its current prefix
//     kp[MAX_KS]         per k: its key prefix so far (8 bits per level)
//     kseg[MAX_KS]       per k: index of its prefix in act[]
//     act[MAX_KS]        the distinct prefixes holding a k, ascending
//     ctl[64]            ctl[0] = number of entries in act[]
//
// A float maps to an order-preserving 32-bit key; four levels of 8-bit digits
// resolve it.  Level L (0..3) is one counting pass over the whole input that
// histograms digit L of every key whose top 8L bits are an active prefix, then
// one single-CTA kernel that moves every k into its child prefix and builds the
// next level's prefix list.  Per call: init + 4 x (count + advance) = 9 launches.
//
// What must be zero: only the histogram rows a counting pass adds into.
// na_init clears row 0 before level 0; na_advance clears rows [0, nact) of the
// next level after it has read this level's rows.  Everything else is written
// before it is read, so the scratch needs no zeroing between calls.

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "ggms_noalloc.h"

namespace ggms_noalloc {

constexpr uint32_t MAXK = GGMS_NOALLOC_MAX_KS;
constexpr uint32_t NBIN = 256;
constexpr uint32_t OFF_HIST = 0;
constexpr uint32_t OFF_KR = OFF_HIST + NBIN * MAXK;
constexpr uint32_t OFF_KP = OFF_KR + MAXK;
constexpr uint32_t OFF_KSEG = OFF_KP + MAXK;
constexpr uint32_t OFF_ACT = OFF_KSEG + MAXK;
constexpr uint32_t OFF_CTL = OFF_ACT + MAXK;
constexpr uint32_t WORDS = OFF_CTL + 64;
static_assert(WORDS * 4u == GGMS_NOALLOC_SCRATCH_BYTES, "scratch layout and its stated size differ");

// The scratch region.  The driver reserves it when it loads this library's
// kernels on a device; it lives as long as the process.
static __device__ __align__(256) uint32_t g_scratch[WORDS];

constexpr int CNT_NT = 512;       // counting pass: CTA size
constexpr int CNT_UNROLL = 4;     // loads in flight per thread
constexpr uint32_t SH_ROWS = 32;  // histogram rows a CTA keeps in shared memory
constexpr int ADV_NT = 1024;      // advance: one CTA, one thread per k
constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr unsigned FULL = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t f32_key(float v) {
  const uint32_t u = __float_as_uint(v);
  return u ^ ((u >> 31) ? 0xFFFFFFFFu : 0x80000000u);
}
__device__ __forceinline__ float key_f32(uint32_t k) {
  return __uint_as_float(k ^ ((k >> 31) ? 0x80000000u : 0xFFFFFFFFu));
}

// The ks travel inside the launch arguments (4 KB; launch arguments may be up
// to 32 KB), so the caller's host array is free when the call returns.
struct KList {
  uint32_t k[MAXK];
};

__global__ __launch_bounds__(ADV_NT) void na_init(const __grid_constant__ KList ks, uint32_t nk, uint32_t n,
                                                  uint32_t* __restrict__ scr) {
  const uint32_t t = threadIdx.x;
  if (t < nk) {
    scr[OFF_KR + t] = n - ks.k[t];  // k-th largest = ascending rank n - k
    scr[OFF_KP + t] = 0u;
    scr[OFF_KSEG + t] = 0u;
  }
  if (t < NBIN) scr[OFF_HIST + t] = 0u;
  if (t == 0) scr[OFF_CTL] = 1u;
}

// Counting pass of level L: hist[s][digit L of key] for every key whose top 8L
// bits equal act[s].  Grid-stride over the input with CNT_UNROLL independent
// loads per thread; equal bins inside a warp are merged (match.any) before the
// atomic add, so heavily repeated digits do not serialise.
template <int L>
__global__ __launch_bounds__(CNT_NT) void na_count(const float* __restrict__ in, uint64_t n,
                                                   uint32_t* __restrict__ scr) {
  __shared__ uint32_t sact[MAXK];
  __shared__ uint32_t bmap[2048];  // one bit per value of the key's top 16 bits
  __shared__ uint32_t shist[SH_ROWS * NBIN];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t nact = (L == 0) ? 1u : scr[OFF_CTL];
  const bool in_smem = nact <= SH_ROWS;
  uint32_t* ghist = scr + OFF_HIST;
  if (L > 0) {
    for (uint32_t i = tid; i < 2048u; i += CNT_NT) bmap[i] = 0u;
    for (uint32_t i = tid; i < nact; i += CNT_NT) sact[i] = scr[OFF_ACT + i];
    __syncthreads();
    for (uint32_t i = tid; i < nact; i += CNT_NT) {
      const uint32_t p = sact[i];
      if (L == 1) {
#pragma unroll
        for (uint32_t w = 0; w < 8; ++w) bmap[p * 8u + w] = FULL;  // top byte p: 256 values of the top 16 bits
      } else {
        const uint32_t q = (L == 2) ? p : (p >> 8);
        atomicOr(&bmap[q >> 5], 1u << (q & 31));
      }
    }
  }
  if (in_smem)
    for (uint32_t i = tid; i < nact * NBIN; i += CNT_NT) shist[i] = 0u;
  __syncthreads();

  const uint64_t stride = (uint64_t)gridDim.x * CNT_NT;
  // b0 is the same for the 32 lanes of a warp, so every lane reaches match.any
  for (uint64_t b0 = (uint64_t)blockIdx.x * CNT_NT + warp * 32u; b0 < n; b0 += CNT_UNROLL * stride) {
    float v[CNT_UNROLL];
#pragma unroll
    for (int j = 0; j < CNT_UNROLL; ++j) {
      const uint64_t i = b0 + lane + (uint64_t)j * stride;
      v[j] = (i < n) ? __ldg(in + i) : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < CNT_UNROLL; ++j) {
      const uint64_t i = b0 + lane + (uint64_t)j * stride;
      uint32_t idx = NONE;
      if (i < n) {
        const uint32_t u = f32_key(v[j]);
        uint32_t s = 0;
        bool hit = true;
        if constexpr (L > 0) {
          const uint32_t t16 = u >> 16;
          hit = (bmap[t16 >> 5] >> (t16 & 31)) & 1u;
          if (hit) {
            const uint32_t p = u >> (32 - 8 * L);
            uint32_t lo = 0, hi = nact - 1;  // largest s with act[s] <= p
            while (lo < hi) {
              const uint32_t mid = (lo + hi + 1) >> 1;
              if (sact[mid] <= p) lo = mid; else hi = mid - 1;
            }
            hit = sact[lo] == p;
            s = lo;
          }
        }
        if (hit) idx = s * NBIN + ((u >> (24 - 8 * L)) & 255u);
      }
      if (in_smem) {  // shared atomics without a return value cost less than a match instruction
        if (idx != NONE) atomicAdd(&shist[idx], 1u);
      } else {  // global atomics: one per distinct counter of the warp
        const uint32_t peers = __match_any_sync(FULL, idx);
        if (idx != NONE && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&ghist[idx], (uint32_t)__popc(peers));
      }
    }
  }
  if (in_smem) {
    __syncthreads();
    for (uint32_t i = tid; i < nact * NBIN; i += CNT_NT) {
      const uint32_t c = shist[i];
      if (c) atomicAdd(&ghist[i], c);
    }
  }
}

// One thread per k: find the bin of the k's rank in its prefix's histogram row,
// extend the prefix by that digit, then number the distinct child prefixes in
// ascending order (a bitmap over (parent, digit) pairs and a popcount scan) as
// the next level's act[].  The last level writes the answers.
template <int L>
__global__ __launch_bounds__(ADV_NT) void na_advance(uint32_t* __restrict__ scr, uint32_t nk,
                                                     float* __restrict__ out) {
  __shared__ uint32_t nb[MAXK * NBIN / 32];  // bit s*256+digit: a k moves into that child
  __shared__ uint32_t tbase[ADV_NT];
  __shared__ uint32_t red[32];
  __shared__ uint32_t total;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (uint32_t w = t; w < MAXK * NBIN / 32; w += ADV_NT) nb[w] = 0u;
  __syncthreads();
  uint32_t s = 0, bin = 0, np = 0;
  if (t < nk) {
    s = scr[OFF_KSEG + t];
    const uint32_t r = scr[OFF_KR + t];
    const uint4* row = reinterpret_cast<const uint4*>(scr + OFF_HIST + s * NBIN);
    uint32_t cum = 0;
    bool found = false;
    // eight batches of 32 bins, 8 independent 16-byte loads each
#pragma unroll 1
    for (uint32_t b = 0; b < 8 && !found; ++b) {
      uint4 q[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) q[j] = row[b * 8 + j];
      uint32_t tot = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) tot += q[j].x + q[j].y + q[j].z + q[j].w;
      if (r < cum + tot) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const uint32_t c4[4] = {q[j].x, q[j].y, q[j].z, q[j].w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if (!found) {
              if (r < cum + c4[e]) {
                found = true;
                bin = b * 32 + j * 4 + e;
              } else {
                cum += c4[e];
              }
            }
          }
        }
      } else {
        cum += tot;
      }
    }
    // the counts of the row sum to the prefix's population, which holds rank r,
    // so `found` is always set here
    np = (scr[OFF_KP + t] << 8) | bin;
    scr[OFF_KR + t] = r - cum;
    scr[OFF_KP + t] = np;
    atomicOr(&nb[(s * NBIN + bin) >> 5], 1u << (bin & 31));
  }
  if (L == 3) {
    if (t < nk) out[t] = key_f32(np);
    return;
  }
  __syncthreads();  // all reads of this level's histogram rows are done
  // exclusive scan of the popcounts, 8 bitmap words per thread
  uint32_t cnt = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) cnt += __popc(nb[t * 8 + w]);
  uint32_t inc = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t x = __shfl_up_sync(FULL, inc, o);
    if ((int)lane >= o) inc += x;
  }
  if (lane == 31) red[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t x = red[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, x, o);
      if ((int)lane >= o) x += y;
    }
    red[lane] = x;
    if (lane == 31) total = x;
  }
  __syncthreads();
  tbase[t] = inc - cnt + (warp ? red[warp - 1] : 0u);
  __syncthreads();
  const uint32_t nact = total;
  if (t < nk) {
    const uint32_t g = s * NBIN + bin, w = g >> 5, grp = w >> 3;
    uint32_t rank = tbase[grp] + __popc(nb[w] & ((1u << (g & 31)) - 1u));
    for (uint32_t x = grp * 8; x < w; ++x) rank += __popc(nb[x]);
    scr[OFF_KSEG + t] = rank;
    scr[OFF_ACT + rank] = np;  // every k of this child writes the same value
  }
  // clear the rows the next counting pass adds into
  uint4* h4 = reinterpret_cast<uint4*>(scr + OFF_HIST);
  for (uint32_t i = t; i < nact * (NBIN / 4); i += ADV_NT) h4[i] = make_uint4(0u, 0u, 0u, 0u);
  if (t == 0) scr[OFF_CTL] = nact;
}

// ------------------------------------------------------------------ host side
constexpr int MAX_DEVICES = 64;
struct DevState {
  uint32_t* scratch;
  int sms;
};
static std::mutex g_mu;
static int g_sms[MAX_DEVICES];

// With the caller's device current: the address of its scratch region and its
// SM count.  The address is looked up on every call (a table lookup once the
// module is loaded; it allocates nothing), so it is never stale -- after a
// cudaDeviceReset the module is reloaded and the region may move.  The SM
// count is kept per device.
static int device_state(DevState* out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return GGMS_E_CUDA;
  if (dev < 0 || dev >= MAX_DEVICES) return GGMS_E_UNSUPPORTED;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return GGMS_E_CUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_sms[dev] <= 0) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
      return GGMS_E_CUDA;
    g_sms[dev] = sms;
  }
  out->scratch = static_cast<uint32_t*>(p);
  out->sms = g_sms[dev];
  return GGMS_OK;
}

}  // namespace ggms_noalloc

extern "C" int ggms_multiselect_noalloc_f32(const float* d_in, int64_t n, const uint32_t* ks,
                                            int32_t num_ks, float* d_out, void* stream) {
  using namespace ggms_noalloc;
  if (!d_in || (reinterpret_cast<uintptr_t>(d_in) & 3u)) return GGMS_E_INVALID_ARG;
  if (n < 1 || n > (int64_t)0xFFFFFFFFu || num_ks < 0) return GGMS_E_INVALID_ARG;
  if (num_ks > (int32_t)MAXK) return GGMS_E_UNSUPPORTED;
  if (num_ks == 0) return GGMS_OK;
  if (!ks || !d_out || (reinterpret_cast<uintptr_t>(d_out) & 3u)) return GGMS_E_INVALID_ARG;
  KList kl;
  for (int32_t i = 0; i < num_ks; ++i) {
    if (ks[i] < 1u || (int64_t)ks[i] > n) return GGMS_E_INVALID_ARG;
    kl.k[i] = ks[i];
  }
  // An error that earlier work left in the runtime belongs to that work: do
  // not launch on top of it, and do not clear it.
  if (cudaPeekAtLastError() != cudaSuccess) return GGMS_E_CUDA;
  DevState ds;
  const int rc = device_state(&ds);
  if (rc != GGMS_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint32_t nk = (uint32_t)num_ks;
  const uint64_t un = (uint64_t)n;
  const int grid = ds.sms * 4;
  na_init<<<1, ADV_NT, 0, st>>>(kl, nk, (uint32_t)n, ds.scratch);
  na_count<0><<<grid, CNT_NT, 0, st>>>(d_in, un, ds.scratch);
  na_advance<0><<<1, ADV_NT, 0, st>>>(ds.scratch, nk, d_out);
  na_count<1><<<grid, CNT_NT, 0, st>>>(d_in, un, ds.scratch);
  na_advance<1><<<1, ADV_NT, 0, st>>>(ds.scratch, nk, d_out);
  na_count<2><<<grid, CNT_NT, 0, st>>>(d_in, un, ds.scratch);
  na_advance<2><<<1, ADV_NT, 0, st>>>(ds.scratch, nk, d_out);
  na_count<3><<<grid, CNT_NT, 0, st>>>(d_in, un, ds.scratch);
  na_advance<3><<<1, ADV_NT, 0, st>>>(ds.scratch, nk, d_out);
  return cudaGetLastError() == cudaSuccess ? GGMS_OK : GGMS_E_CUDA;
}
