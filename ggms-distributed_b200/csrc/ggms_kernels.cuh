// ggms_kernels.cuh -- device kernels of the exact multiselect engine.
//
// Pipeline for one vector (all on the device, no host round trip):
//   k_init        ks (1-based k-th largest) -> 0-based ascending ranks
//   asg_*         draw S sample keys, sort them, build the level-0 assigner
//   l0_count      PASS 1 over the input: per-CTA shared histogram of buckets
//   l0_scan       inclusive scan of the bucket counts
//   l0_locate     each k finds its bucket and its rank inside the bucket
//   l0_children   active buckets -> key range (inverse of the assigner);
//                 single-key buckets resolve their ks at once, the others
//                 become refinement segments
//   l0_relabel    ks follow their bucket
//   l0_compact    PASS 2 over the input: copy the keys of refinement segments
//   lvl_* (x L)   the same steps over candidates only, with radix bins of
//                 11 key bits, until every k sits in a single-key bin
//   write_out     answers (as the caller's type) in the caller's k order
//
// Reference steps these replace (DistributedSMOS/bucketMultiselect.cu):
//   minmax (:543-547) -- not needed: the assigner has open tail buckets;
//   k sort + peel (:625-656) -- not needed: ks are located independently;
//   generatePivots (:421-515) -> asg_*;  assignSmartBucket (:135-210) -> l0_count;
//   sumCounts (:219-226) -> l0_scan;  findKBuckets (:92-116, host) -> l0_locate;
//   unique buckets + reindexCounts (:726-768, host + kernel) -> l0_children;
//   copyElements (:254-313) -> l0_compact;  thrust::sort + copyValuesInChunk
//   (:814-833) -> the refinement levels + write_out.
// IterativeSMOS (DistributedSMOS/iterativeSMOS.cu:1348-1531) repeats
// bucketing over the survivors with re-fitted pivots; here the survivors are
// refined with exact radix bins of the known key range, which ends in a bounded
// number of levels (3 for 32-bit keys, 6 for 64-bit) with every k exact.
#pragma once
#include <cooperative_groups.h>

#include "ggms_internal.cuh"
#include "../../include/ggms.h"

GGMS_BEGIN

constexpr unsigned FULL = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t warp_incl_scan_u32(uint32_t v, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if ((int)lane >= o) v += t;
  }
  return v;
}

__device__ __forceinline__ void set_status(Counters* C, uint32_t code) {
  atomicCAS(&C->status, 0u, code);
}

// streaming 16-byte load that does not allocate in L1 (each byte is read once per pass)
__device__ __forceinline__ uint4 ld_stream16(const void* p) {
  uint4 r;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p));
  return r;
}

// splitmix64 finaliser (Steele, Lea, Flood 2014) -- sample positions
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <typename K> __host__ __device__ constexpr K key_max() { return (K)~(K)0; }

// ------------------------------------------------------------------ block scan (1024 threads)
// Inclusive scan of `cnt` (multiple of NT) uint32 values in shared or global
// memory, in place.  Returns (to thread 0) the maximum element.  Warp w scans
// the contiguous chunk [w * cnt/32, (w + 1) * cnt/32) row by row (lane l holds
// element 32 i + l of row i), so every access of a warp is 32 consecutive
// words: no bank conflicts in shared memory, coalesced in global memory.
template <int NT>
__device__ void block_inclusive_scan_global(uint32_t* data, uint32_t cnt, uint32_t* smem_warp,
                                            uint32_t* max_out) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t rows = cnt / NT;  // rows of 32 per warp
  uint32_t* chunk = data + (size_t)warp * rows * 32u;
  uint32_t sum = 0, mx = 0;
  for (uint32_t i = 0; i < rows; ++i) {
    const uint32_t v = chunk[i * 32u + lane];
    mx = max(mx, v);
    sum += v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_xor_sync(FULL, sum, o);
    mx = max(mx, __shfl_xor_sync(FULL, mx, o));
  }
  if (lane == 0) {
    smem_warp[warp] = sum;
    smem_warp[32 + warp] = mx;
  }
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < NT / 32) ? smem_warp[lane] : 0u;
    uint32_t wm = (lane < NT / 32) ? smem_warp[32 + lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(FULL, w, o);
      if (lane >= o) w += t;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wm = max(wm, __shfl_xor_sync(FULL, wm, o));
    smem_warp[lane] = w;  // inclusive warp totals
    if (lane == 0) smem_warp[64] = wm;
  }
  __syncthreads();
  uint32_t carry = warp > 0 ? smem_warp[warp - 1] : 0u;
  for (uint32_t i = 0; i < rows; ++i) {
    const uint32_t inc = warp_incl_scan_u32(chunk[i * 32u + lane], lane);
    chunk[i * 32u + lane] = carry + inc;
    carry += __shfl_sync(FULL, inc, 31);
  }
  if (tid == 0 && max_out) *max_out = smem_warp[64];
  __syncthreads();
}

// Zeroes up to three ranges of 32-bit words (a null range is skipped): the
// level-0 histogram, flags and k counts, and the windows when there are none.
// In the kernel chain instead of memset nodes, which would end the chain's
// programmatic launches.
__global__ void zero_words(uint32_t* a, uint32_t na, uint32_t* b, uint32_t nb, uint32_t* c, uint32_t nc) {
  pdl_entry();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
  for (uint32_t i = t; i < na; i += st) a[i] = 0u;
  for (uint32_t i = t; i < nb; i += st) b[i] = 0u;
  if (c)
    for (uint32_t i = t; i < nc; i += st) c[i] = 0u;
}

// ------------------------------------------------------------------ ks
// 1-based k-th largest -> 0-based rank in ascending order (the reference's
// wrappers compute length - k + 1, 1-based smallest: bucketMultiselect.cu:860-861).
__global__ void k_init_single(const uint32_t* __restrict__ ks, uint32_t nk, uint64_t n,
                              uint32_t* k_rank, uint32_t* k_seg, Counters* C) {
  pdl_entry();
  GGMS_TRACE(0);
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nk) return;
  uint32_t k = ks[i];
  if (k < 1u || (uint64_t)k > n) {
    set_status(C, GGMS_E_INVALID_ARG);
    k_seg[i] = K_DONE;
    k_rank[i] = 0;
    return;
  }
  k_rank[i] = (uint32_t)(n - k);
  k_seg[i] = 0;
}

// top-k: k_i = i + 1 (the (i+1)-th largest), i.e. ascending rank n - 1 - i
__global__ void k_init_topk(uint32_t nk, uint64_t n, uint32_t* k_rank, uint32_t* k_seg) {
  pdl_entry();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nk) return;
  k_rank[i] = (uint32_t)(n - 1u - i);
  k_seg[i] = 0;
}

// ------------------------------------------------------------------ sampling
template <typename T>
__global__ void asg_sample(const T* __restrict__ in, uint64_t n, uint32_t S, uint64_t seed,
                           typename KeyOf<T>::K* out) {
  pdl_entry();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S) return;
  uint64_t h = mix64(seed ^ mix64((uint64_t)i + 0x632BE59BD9B4E019ull));
  uint64_t pos = __umul64hi(h, n);  // uniform in [0, n)
  out[i] = KeyOf<T>::to(in[pos]);
}

// Bitonic sort of one chunk of CH keys per CTA in shared memory.
template <typename K, int CH, int NT>
__global__ __launch_bounds__(NT) void asg_sort_chunks(const K* __restrict__ in, K* out, uint32_t S) {
  pdl_entry();
  __shared__ K s[CH];
  const uint32_t base = blockIdx.x * CH;
  const uint32_t cnt = min((uint32_t)CH, S - base);
  for (uint32_t i = threadIdx.x; i < CH; i += NT) s[i] = i < cnt ? in[base + i] : key_max<K>();
  __syncthreads();
  for (uint32_t k = 2; k <= (uint32_t)CH; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < (uint32_t)CH; i += NT) {
        uint32_t ixj = i ^ j;
        if (ixj > i) {
          K a = s[i], b = s[ixj];
          bool up = (i & k) == 0;
          if ((a > b) == up) {
            s[i] = b;
            s[ixj] = a;
          }
        }
      }
      // a stage with j < 32 pairs keys of one warp only (i and i ^ j belong to
      // lanes l and l ^ j): a warp barrier suffices unless the next stage
      // reaches across warps
      const uint32_t nj = j > 1 ? (j >> 1) : k;  // the next stage's j
      if (nj >= 32u || (j == 1 && k == (uint32_t)CH)) __syncthreads(); else __syncwarp();
    }
  }
  for (uint32_t i = threadIdx.x; i < cnt; i += NT) out[base + i] = s[i];
}

// Sort of a drawn sample (S >= 1024 * CTAS keys, asg_sample drew it: a wide
// grid reaches the random positions far faster than a few SMs would) in one
// launch of one thread-block cluster of CTAS = 8 or 16 CTAs (16 is a
// non-portable cluster size: used when the device can place one, so that each
// warp ranks half as many keys).  CTA c loads sample keys [c * S/CTAS,
// (c + 1) * S/CTAS) into its shared memory; then an LSD radix sort with 8-bit
// digits runs over the whole cluster.  Per digit pass:
//   1. every warp ranks its keys stably, 32 at a time: each lane ORs its bit
//      into a per-warp lane mask of its digit (a shared atomic), reads the mask
//      back and counts the lanes below it; the lowest lane of the digit adds
//      the group to the warp's digit count and clears the mask.  A warp whose
//      32 keys share one digit skips the atomics.  (Measured on the B200 for
//      4096 keys per SM: 1.3 us per pass with diverse digits, against 2.2 us
//      for eight ballots and 4.2 us for a match instruction.);
//   2. every CTA pushes its 256 digit counts into a table in each peer's
//      shared memory (distributed shared memory stores); after a cluster
//      barrier every CTA reads, from its own table, where its keys of each
//      digit start, both in its own digit-grouped order and in the cluster's
//      next order;
//   3. each CTA groups its keys by digit in its own shared memory (random
//      stores stay on the SM);
//   4. each CTA copies its grouped keys to their owners: thread i moves key i,
//      so a warp's 32 stores go to consecutive positions of one or two digit
//      runs -- whole lines over the SM-to-SM network instead of one 4- or
//      8-byte transaction per key.
// Two cluster barriers per pass: counts visible (before 2) and the next order
// complete (after 4); every key is read out of the current order in step 1,
// before the first barrier, so step 4 may overwrite it.  A pass in which every key has the same digit is skipped (the permutation is
// the identity).  4 passes for 32-bit keys, 8 for 64-bit ones; the sorted
// sample is written out with coalesced stores.
namespace cgx = cooperative_groups;
constexpr int CS_NT = 1024;
__host__ __device__ constexpr uint32_t cs_min_s(int ctas) { return (uint32_t)ctas * CS_NT; }  // 1 key per thread

template <typename K, int CTAS>
struct ClusterSortSmem {
  static constexpr uint32_t PER = 65536u / CTAS;  // keys per CTA at S = 65536
  K a[PER];                        // this CTA's share of the current order
  K b[PER];                        // this CTA's keys grouped by the pass's digit
  uint32_t hist[CS_NT / 32][256];  // per warp: digit counts, then their prefixes over the warps
  uint32_t pmask[CS_NT / 32][256]; // per warp: lanes of the current round holding the digit
  uint32_t ctab[CTAS][256];        // every CTA's digit counts (written by that CTA)
  uint32_t ccnt[256];              // this CTA's digit counts
  uint32_t gbase[256];             // first position of (digit, this CTA) in the next order
  uint32_t lbase[256];             // first position of the digit in b
  uint32_t red[2][8];
  uint32_t skip;
};

// Launched with a cluster dimension of CTAS (launch_sort_cluster).
template <typename K, int CTAS>
__global__ void __launch_bounds__(CS_NT) asg_sort_cluster(const K* __restrict__ drawn, uint32_t S, K* sorted) {
  pdl_entry();
  using Smem = ClusterSortSmem<K, CTAS>;
  constexpr int KB = (int)sizeof(K) * 8;
  constexpr int KPT_MAX = (int)(Smem::PER / CS_NT);    // 8 or 4
  extern __shared__ __align__(128) uint8_t smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  cgx::cluster_group cluster = cgx::this_cluster();
  const uint32_t me = cluster.block_rank();
  const uint32_t per = S / CTAS;                       // keys per CTA: a power of two
  const uint32_t per_sh = (uint32_t)__ffs((int)per) - 1u;
  const uint32_t kpt = per / CS_NT;                    // keys per thread
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // warp w owns positions [w * 32 * kpt, (w + 1) * 32 * kpt) of this CTA's
  // share; in round r its lane l holds position w * 32 * kpt + r * 32 + l
  const uint32_t wbase = warp * 32u * kpt;
  GGMS_TRACE(1);
  K* A = sm.a;
  for (uint32_t i = tid; i < per; i += CS_NT) A[i] = drawn[(size_t)me * per + i];
  for (uint32_t d = lane; d < 256u; d += 32u) sm.pmask[warp][d] = 0u;
  __syncthreads();
  const uint32_t lt = lanemask_lt();
  for (int sh = 0; sh < KB; sh += 8) {
    for (uint32_t d = lane; d < 256u; d += 32u) sm.hist[warp][d] = 0u;
    __syncwarp();
    K key[KPT_MAX];
    uint32_t dg[KPT_MAX], off[KPT_MAX];
#pragma unroll
    for (int r = 0; r < KPT_MAX; ++r) {
      if ((uint32_t)r >= kpt) break;
      key[r] = A[wbase + r * 32u + lane];
      const uint32_t d = (uint32_t)(key[r] >> sh) & 255u;
      const bool one = __all_sync(FULL, d == __shfl_sync(FULL, d, 0));
      if (!one) {
        atomicOr(&sm.pmask[warp][d], 1u << lane);
        __syncwarp();
      }
      const uint32_t peers = one ? FULL : sm.pmask[warp][d];
      const uint32_t base = sm.hist[warp][d];
      __syncwarp();
      if ((peers & lt) == 0u) {  // the lowest lane of the group
        sm.hist[warp][d] = base + __popc(peers);
        if (!one) sm.pmask[warp][d] = 0u;
      }
      __syncwarp();
      dg[r] = d;
      off[r] = base + __popc(peers & lt);
    }
    __syncthreads();
    if (sh < 24) GGMS_TRACE(46 + (sh >> 3) * 4);
    // per digit: exclusive prefix over the warps (in place) and this CTA's total
    {
      const uint32_t d = tid >> 2, q = tid & 3u;       // 4 threads per digit, 8 warps each
      uint32_t c[8], sum = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) { c[j] = sm.hist[q * 8 + j][d]; sum += c[j]; }
      uint32_t inc = sum;
#pragma unroll
      for (int o = 1; o < 4; o <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, inc, o);
        if ((int)q >= o) inc += t;
      }
      uint32_t run = inc - sum;
#pragma unroll
      for (int j = 0; j < 8; ++j) { sm.hist[q * 8 + j][d] = run; run += c[j]; }
      if (q == 3u) sm.ccnt[d] = inc;
    }
    __syncthreads();
    for (uint32_t i = tid; i < 256u * CTAS; i += CS_NT)  // row `me` of every peer's table
      *cluster.map_shared_rank(&sm.ctab[me][i & 255u], i >> 8) = sm.ccnt[i & 255u];
    cluster.sync();  // (1) every CTA's digit counts are in every table
    if (tid < 256u) {
      uint32_t tot = 0, before = 0;
#pragma unroll
      for (int c = 0; c < CTAS; ++c) {
        const uint32_t v = sm.ctab[c][tid];
        tot += v;
        before += ((uint32_t)c < me) ? v : 0u;
      }
      const uint32_t mine = sm.ccnt[tid];
      // exclusive scans over the 256 digits (8 warps): the totals and this CTA's counts
      const uint32_t inc_t = warp_incl_scan_u32(tot, lane);
      const uint32_t inc_m = warp_incl_scan_u32(mine, lane);
      if (lane == 31) {
        sm.red[0][warp] = inc_t;
        sm.red[1][warp] = inc_m;
      }
      if (tid == 0) sm.skip = 0u;
      asm volatile("bar.sync 1, 256;" ::: "memory");
      uint32_t pre_t = inc_t - tot, pre_m = inc_m - mine;
      for (uint32_t w = 0; w < warp; ++w) {
        pre_t += sm.red[0][w];
        pre_m += sm.red[1][w];
      }
      sm.gbase[tid] = pre_t + before;
      sm.lbase[tid] = pre_m;
      if (tot == S) sm.skip = 1u;  // every key has this digit: nothing moves
    }
    __syncthreads();
    if (sh < 24) GGMS_TRACE(47 + (sh >> 3) * 4);
    const bool skip = sm.skip != 0u;
    if (!skip) {
#pragma unroll
      for (int r = 0; r < KPT_MAX; ++r) {
        if ((uint32_t)r >= kpt) break;
        sm.b[sm.lbase[dg[r]] + sm.hist[warp][dg[r]] + off[r]] = key[r];
      }
    }
    __syncthreads();  // b is complete (the cluster's a was read into registers before (1))
    if (sh < 24) GGMS_TRACE(48 + (sh >> 3) * 4);
    if (!skip) {
      for (uint32_t i = tid; i < per; i += CS_NT) {
        const K k = sm.b[i];
        const uint32_t d = (uint32_t)(k >> sh) & 255u;
        const uint32_t pos = sm.gbase[d] + (i - sm.lbase[d]);
        *cluster.map_shared_rank(&A[pos & (per - 1u)], pos >> per_sh) = k;
      }
    }
    cluster.sync();  // (2) the next order is complete; the counts have been read
    if (sh < 24) GGMS_TRACE(49 + (sh >> 3) * 4);
  }
  K* out = sorted + (size_t)me * per;
  for (uint32_t i = tid; i < per; i += CS_NT) out[i] = A[i];
  GGMS_TRACE(2);
}

template <typename K>
__device__ __forceinline__ AsgView<K> asg_view_global(const Assigner<K>* A) {
  AsgView<K> v;
  v.x = A->x; v.base = A->base; v.slope = A->slope; v.idx = A->idx;
  v.M = A->M; v.B = A->B; v.csh = A->csh;
  return v;
}

// ------------------------------------------------------------------ level 0 (one vector)
template <typename K>
__device__ __forceinline__ GridView<K> grid_view_global(const Grid<K>* G) {
  GridView<K> v;
  v.t1 = G->t1; v.t2 = G->t2; v.origin = G->origin; v.gmax = G->gmax;
  v.sh1 = G->sh1; v.B = G->B;
  return v;
}

// Copy the grid into shared memory (t1: GRID_T1 entries, t2: GRID_SUBCAP).
template <typename K>
__device__ __forceinline__ GridView<K> grid_to_smem(const Grid<K>* __restrict__ G, uint2* s1, uint2* s2) {
  const uint32_t nc = G->ncell, ns = G->nsubent;
  // both tables as one index range, 8 loads in flight per thread
  const uint32_t tot = nc + ns, nt = blockDim.x;
  for (uint32_t i0 = threadIdx.x; i0 < tot; i0 += 8u * nt) {
    uint2 v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t i = i0 + (uint32_t)u * nt;
      if (i < tot) v[u] = i < nc ? G->t1[i] : G->t2[i - nc];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t i = i0 + (uint32_t)u * nt;
      if (i < tot) {
        if (i < nc) s1[i] = v[u];
        else s2[i - nc] = v[u];
      }
    }
  }
  GridView<K> v;
  v.t1 = s1; v.t2 = s2; v.origin = G->origin; v.gmax = G->gmax;
  v.sh1 = G->sh1; v.B = G->B;
  return v;
}

constexpr size_t GRID_SMEM = sizeof(uint2) * (GRID_T1 + GRID_SUBCAP);

// 16-byte vector view of the input
template <typename T> struct Vec16 {
  static constexpr int N = 16 / sizeof(T);
};

template <typename T>
__device__ __forceinline__ void unpack16(const uint4& q, T (&e)[Vec16<T>::N]) {
  static_assert(sizeof(T) * Vec16<T>::N == 16, "");
  __builtin_memcpy(e, &q, 16);
}

// The passes run 1024 threads per SM at least (2 CTAs of 512, 4 of 256, 1 of
// 1024): the register budget is 64 per thread, which the launch bounds state
// so that the compiler neither exceeds it nor spills well below it.
#define PASS_MIN_CTAS(nt) ((nt) >= 1024 ? 1 : 1024 / (nt))

// Per-warp queues of the passes.  Keys that need the long path (bucket
// computation) are spread over the input; handling each where it is found
// would run the long path for every warp that holds one.  They are appended
// to a per-warp queue in shared memory instead and handled 32 at a time, one
// per lane.
constexpr uint32_t WQ_DEPTH = 64;  // per-warp queue slots: < 32 waiting + 32 appended

__host__ __device__ constexpr uint32_t wq_bytes(uint32_t nt, uint32_t key_bytes) {
  return (nt / 32) * WQ_DEPTH * key_bytes;
}

// Appends the flagged keys of the warp to its queue (qn: warp-uniform fill).
// Returns true (for the whole warp) when 32 keys were waiting: they are taken
// off the queue, one per lane, into *out.  All 32 lanes must call it.
template <typename K>
__device__ __forceinline__ bool wq_push(K* wq, uint32_t& qn, bool flag, K key, uint32_t lane, K* out) {
  const uint32_t m = __ballot_sync(FULL, flag);
  if (!m) return false;
  if (flag) wq[qn + __popc(m & ((1u << lane) - 1u))] = key;
  qn += __popc(m);
  if (qn < 32u) return false;
  __syncwarp();
  *out = wq[lane];
  const K k1 = (lane + 32u < qn) ? wq[lane + 32u] : (K)0;
  __syncwarp();
  if (lane + 32u < qn) wq[lane] = k1;
  qn -= 32u;
  return true;
}

// Key test of the windowed passes: is the key inside one of R key ranges
// [lo, lo + sp]; with CNT, also count per range the keys below its first key.
template <typename K, uint32_t R, bool CNT>
struct RunTest {
  K lo[R], sp[R];
  uint32_t bl[R];
  __device__ __forceinline__ bool operator()(K k) {
    bool h = false;
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) {
      if (CNT) bl[r] += k < lo[r] ? 1u : 0u;
      h = h | ((K)(k - lo[r]) <= sp[r]);
    }
    return h;
  }
};

// ------------------------------------------------------------------ input streams of the passes
// The body of the input (16-byte vectors from its first 16-byte boundary) is
// split between the CTAs the same way in PASS 1 and PASS 2, so that PASS 2's
// per-CTA write ranges (sized by PASS 1) fit.  Three ways to stream it (the
// template parameter UNROLL of the pass kernels):
//   UNROLL > 0:  grid-strided rounds of UNROLL non-allocating vector loads per
//                thread, into registers;
//   UNROLL == -1 (TMA ring): chunks of RING_VECS vectors (32 KB) dealt
//                round-robin to the CTAs and staged in a ring of shared-memory
//                stages: thread 0 fills a stage with one bulk copy
//                (cp.async.bulk, the TMA engine) that completes on the stage's
//                "full" mbarrier; every thread reads its V vectors back and
//                each warp then arrives on the stage's "empty" mbarrier.
//                Thread 0 refills every released stage as it passes by and
//                blocks only when the chunk it needs itself is not issued yet;
//   UNROLL == -2 (async copies): chunks of 1024 vectors (16 KB) dealt
//                round-robin to the CTAs; every thread copies its own vectors
//                of the next ASYNC_D - 1 chunks into its private shared-memory
//                slots with cp.async and waits only for its own oldest group:
//                no barrier between threads at all.
// Every thread of a CTA handles the same number of vectors in all three, so
// the warps stay converged.  The vectors past the main part (main_end ..
// nvec) are left to the caller, one per thread, grid-strided.
constexpr uint32_t RING_BYTES = 32768;
constexpr uint32_t RING_VECS = RING_BYTES / 16;
constexpr uint32_t RING_MAX_ST = 8;
constexpr uint32_t ASYNC_VECS = 1024;   // vectors of one async-copy chunk (16 KB)
constexpr int ASYNC_D = 4;              // async-copy chunks per thread in shared memory

struct RingBars {
  unsigned long long full[RING_MAX_ST];
  unsigned long long empty[RING_MAX_ST];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0u;
}
// Non-blocking test of the same.
__device__ __forceinline__ bool mbar_test(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0u;
}
// Waits until the phase of parity `parity` of barrier `a` has completed; gives
// up (false) after about a second, so that a broken pipeline cannot hang the GPU.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity) {
  if (mbar_try(a, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try(a, parity))
    if (clock64() - t0 > (2ll << 30)) return false;
  return true;
}
// One bulk copy global -> this CTA's shared memory, completing on mbarrier `bar`
// (both addresses 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// One 16-byte asynchronous copy global -> shared (L2 only), in the thread's current group.
__device__ __forceinline__ void async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// The TMA ring of one CTA.  All threads call start() and next(); next() is
// CTA-uniform (every thread sees the same chunk count).
template <int NT>
struct Ring {
  static constexpr int V = (int)(RING_VECS / NT);  // vectors per thread per chunk
  const uint4* body;
  uint4* stage0;
  uint32_t bars, nst, nmine, j, issued, G, b;
  bool ok;

  __device__ __forceinline__ uint32_t full(uint32_t s) const { return bars + 8u * s; }
  __device__ __forceinline__ uint32_t empty(uint32_t s) const { return bars + 8u * (RING_MAX_ST + s); }
  // thread 0: this CTA's chunk jj into stage jj % nst
  __device__ __forceinline__ void issue(uint32_t jj) {
    const uint32_t s = jj % nst;
    const uint64_t c = (uint64_t)b + (uint64_t)jj * G;
    mbar_expect_tx(full(s), RING_BYTES);
    bulk_g2s(smem_u32(stage0 + (size_t)s * RING_VECS), body + c * RING_VECS, RING_BYTES, full(s));
  }
  __device__ __forceinline__ void start(const uint4* body_, uint64_t nch, uint4* ring, RingBars* rb,
                                        uint32_t nst_) {
    body = body_;
    stage0 = ring;
    bars = smem_u32(rb);
    nst = min(max(nst_, 2u), RING_MAX_ST);
    G = gridDim.x;
    b = blockIdx.x;
    nmine = nch > b ? (uint32_t)((nch - b + G - 1) / G) : 0u;
    j = 0;
    issued = 0;
    ok = true;
    if (threadIdx.x == 0) {
      for (uint32_t s = 0; s < nst; ++s) {
        mbar_init(full(s), 1u);
        mbar_init(empty(s), NT / 32);
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (; issued < min(nst, nmine); ++issued) issue(issued);
  }
  // This thread's V vectors of the CTA's next chunk; false when the CTA has
  // none left, or (warp-uniformly) after a wait gave up.
  __device__ __forceinline__ bool next(uint4 (&q)[V]) {
    if (j >= nmine || !ok) return false;
    bool good = true;
    if (threadIdx.x == 0) {
      // refill every stage the warps have released (without waiting), and
      // block only when the chunk needed now has not been issued
      while (issued < nmine) {
        const uint32_t jp = issued - nst;  // the chunk the stage held before
        if (issued > j && !mbar_test(empty(jp % nst), (jp / nst) & 1u)) break;
        if (!mbar_wait(empty(jp % nst), (jp / nst) & 1u)) {
          good = false;
          break;
        }
        issue(issued);
        ++issued;
      }
    }
    const uint32_t s = j % nst;
    if (good) good = mbar_wait(full(s), (j / nst) & 1u);
    if (__all_sync(FULL, good)) {
      const uint4* st = stage0 + (size_t)s * RING_VECS;
#pragma unroll
      for (int v = 0; v < V; ++v) q[v] = st[threadIdx.x + v * NT];
      __syncwarp();
      if ((threadIdx.x & 31u) == 0u) mbar_arrive(empty(s));
    } else {
      good = false;
    }
    ok = __all_sync(FULL, good);
    ++j;
    return ok;
  }
  // After the main loop (all threads): with a wait that gave up anywhere, the
  // status is set and thread 0 waits (bounded) for the copies it issued that
  // were not consumed, so none is still writing when the CTA exits.
  __device__ __forceinline__ void finish(Counters* C) {
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicCAS(&C->status, 0u, (uint32_t)GGMS_E_INTERNAL);
        for (uint32_t jj = 0; jj < issued; ++jj)
          if (jj + nst >= issued) mbar_wait(full(jj % nst), (jj / nst) & 1u);
      }
    }
  }
};

// The async-copy pipeline of one thread (UNROLL == -2).
template <int NT>
struct AsyncPipe {
  static constexpr int V = (int)(ASYNC_VECS / NT);  // vectors per thread per chunk
  const uint4* body;
  uint4* slots;  // [ASYNC_D][ASYNC_VECS] vectors, this thread's at tid + v * NT
  uint32_t nmine, j, G, b;
  __device__ __forceinline__ void load(uint32_t jj) {
    const uint64_t c = (uint64_t)b + (uint64_t)jj * G;
    const uint32_t sl = jj % ASYNC_D;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const uint32_t x = threadIdx.x + v * NT;
      async16(smem_u32(slots + (size_t)sl * ASYNC_VECS + x), body + c * ASYNC_VECS + x);
    }
  }
  __device__ __forceinline__ void start(const uint4* body_, uint64_t nch, uint4* slots_) {
    body = body_;
    slots = slots_;
    G = gridDim.x;
    b = blockIdx.x;
    nmine = nch > b ? (uint32_t)((nch - b + G - 1) / G) : 0u;
    j = 0;
    for (uint32_t jj = 0; jj + 1 < (uint32_t)ASYNC_D; ++jj) {
      if (jj < nmine) load(jj);
      async_commit();
    }
  }
  __device__ __forceinline__ bool next(uint4 (&q)[V]) {
    if (j >= nmine) {
      async_wait<0>();
      return false;
    }
    // the slot chunk j + D - 1 goes to was read in the previous call
    if (j + ASYNC_D - 1 < nmine) load(j + ASYNC_D - 1);
    async_commit();
    async_wait<ASYNC_D - 1>();  // this thread's copies of chunk j have landed
    const uint4* sl = slots + (size_t)(j % ASYNC_D) * ASYNC_VECS;
#pragma unroll
    for (int v = 0; v < V; ++v) q[v] = sl[threadIdx.x + v * NT];
    ++j;
    return true;
  }
};

// vectors of one chunk of a staged stream
__host__ __device__ constexpr uint32_t stream_chunk_vecs(int unroll) {
  return unroll == -1 ? RING_VECS : ASYNC_VECS;
}

// The main loop's driver for one pass kernel: run(f) calls f(vector) for each
// of this thread's vectors of the main part.  run() (or next_batch()) is used
// by all threads or none (the kernels branch on CTA-uniform values only); the
// staging starts inside it, so a kernel that skips the main part has no copy
// in flight.
template <int NT, int UNROLL>
struct PassStream {
  static constexpr bool RING = UNROLL == -1, ASYNC = UNROLL == -2;
  static constexpr int V = RING ? Ring<NT>::V : AsyncPipe<NT>::V;
  const uint4* body;
  uint4* ring_smem;
  RingBars* rb;
  uint64_t nvec, nch, gtid, gstride, main_end, rounds;
  uint32_t nst;
  bool started;
  Ring<NT> ring;
  AsyncPipe<NT> pipe;
  __device__ __forceinline__ void start(const uint4* body_, uint64_t nvec_, uint4* ring_smem_, RingBars* rb_,
                                        uint32_t nst_) {
    body = body_;
    nvec = nvec_;
    ring_smem = ring_smem_;
    rb = rb_;
    nst = nst_;
    started = false;
    gtid = (uint64_t)blockIdx.x * NT + threadIdx.x;
    gstride = (uint64_t)gridDim.x * NT;
    if constexpr (UNROLL > 0) {
      rounds = nvec / (gstride * UNROLL);
      main_end = rounds * gstride * UNROLL;
    } else {
      nch = nvec / stream_chunk_vecs(UNROLL);
      main_end = nch * stream_chunk_vecs(UNROLL);
    }
  }
  __device__ __forceinline__ void begin() {
    if constexpr (RING) ring.start(body, nch, ring_smem, rb, nst);
    if constexpr (ASYNC) pipe.start(body, nch, ring_smem);
    started = true;
  }
  __device__ __forceinline__ bool next(uint4 (&q)[V]) {
    if constexpr (RING) return ring.next(q);
    else return pipe.next(q);
  }
  template <typename F>
  __device__ __forceinline__ void run(F&& f) {
    if constexpr (UNROLL > 0) {
      const uint4* vp = body + gtid;
      for (uint64_t r = 0; r < rounds; ++r, vp += gstride * UNROLL) {
        uint4 q[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) q[u] = ld_stream16(vp + u * gstride);
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) f(q[u]);
      }
    } else {
      begin();
      uint4 q[V];
      while (next(q)) {
#pragma unroll
        for (int v = 0; v < V; ++v) f(q[v]);
      }
    }
  }
  // Staged streams only: this thread's vectors of the CTA's next DU / V chunks
  // into q; returns how many it wrote (CTA-uniform; 0 at the end).
  template <int DU>
  __device__ __forceinline__ int next_batch(uint4 (&q)[DU]) {
    static_assert(DU % V == 0, "a batch holds whole chunks");
    if (!started) begin();
    int got = 0;
#pragma unroll
    for (int c = 0; c < DU / V; ++c) {
      uint4 t[V];
      if (!next(t)) break;
#pragma unroll
      for (int v = 0; v < V; ++v) q[c * V + v] = t[v];
      got += V;
    }
    return got;
  }
  // All threads, after the main part (a no-op when the staging never started).
  __device__ __forceinline__ void finish(Counters* C) {
    if constexpr (RING) {
      if (started) ring.finish(C);
    }
    if constexpr (ASYNC) async_wait<0>();
  }
  // vectors of the main part this thread handles
  __device__ __forceinline__ uint64_t my_vecs() const {
    if constexpr (UNROLL > 0) {
      return rounds * UNROLL;
    } else {
      const uint64_t G = gridDim.x, b = blockIdx.x;
      return (nch > b ? (nch - b + G - 1) / G : 0) * (uint64_t)V;
    }
  }
};

// Shared-memory bytes of a pass kernel's staging (0 for the register streams;
// nst: stages of the TMA ring).
__host__ __device__ constexpr size_t ring_bytes(int unroll, uint32_t nst) {
  return unroll == -1 ? (size_t)nst * RING_BYTES + 128
                      : unroll == -2 ? (size_t)ASYNC_D * ASYNC_VECS * 16 + 128 : 0;
}
// The ring's place: the end of the kernel's dynamic shared memory, 128-byte aligned.
__device__ __forceinline__ uint4* ring_at(uint8_t* smem, size_t used) {
  return reinterpret_cast<uint4*>(smem + ((used + 127) & ~(size_t)127));
}

// The uniform main loop's per-vector step: keys that pass test(key) go through
// the per-warp queue to take(key), 32 at a time; the queue's leftovers (qn < 32)
// stay for the caller.
template <typename T, typename Src, typename Test, typename Take>
__device__ __forceinline__ void stream_keys(Src& src, typename KeyOf<T>::K* wq, uint32_t& qn, uint32_t lane,
                                            Test& test, Take&& take) {
  using K = typename KeyOf<T>::K;
  constexpr int EPV = Vec16<T>::N;
  src.run([&](const uint4& qv) {
    T e[EPV];
    unpack16<T>(qv, e);
    K kk[EPV];
    bool hh[EPV];
    bool any = false;
#pragma unroll
    for (int t = 0; t < EPV; ++t) {
      kk[t] = KeyOf<T>::to(e[t]);
      hh[t] = test(kk[t]);
      any = any || hh[t];
    }
    if (!__any_sync(FULL, any)) return;
#pragma unroll
    for (int t = 0; t < EPV; ++t) {
      K k0;
      if (wq_push(wq, qn, hh[t], kk[t], lane, &k0)) take(k0);
    }
  });
}

// Float input: the run tests on the raw bits.  The key of a float is its bits
// with the sign bit flipped (non-negative values) or all bits flipped
// (negative ones), so a key run [lo, lo + sp] that lies within one sign is the
// raw range [lo ^ 2^31, ... + sp] (non-negative) or [~(lo + sp), ... + sp]
// (negative), of the same span; the unsigned test (raw - rlo) <= sp rejects
// every float of the other sign by wrap-around (rlo + sp stays below 2^31, or
// the range ends at 2^32 - 1 - lo).  NaN and +-Inf keep their places.  A run
// over both signs is still one cyclic raw range when it reaches an end of the
// key space: from key 0 it holds every negative float (raw 2^31 .. 2^32 - 1)
// and the non-negative ones up to hi (raw 0 .. hi ^ 2^31); up to the largest
// key it holds every non-negative float and the negative ones down to lo (raw
// 0 .. ~lo).  Returns false for a run over both signs that reaches neither end.
__device__ __forceinline__ bool run_to_raw(uint32_t lo, uint32_t sp, uint32_t& rlo, uint32_t& rsp) {
  const uint32_t hi = lo + sp;
  rsp = sp;
  if (lo >= 0x80000000u) { rlo = lo ^ 0x80000000u; return true; }
  if (hi < 0x80000000u) { rlo = ~hi; return true; }
  if (lo == 0u) { rlo = 0x80000000u; rsp = 0x80000000u + (hi ^ 0x80000000u); return true; }
  if (hi == 0xFFFFFFFFu) { rlo = 0u; rsp = ~lo; return true; }
  return false;
}
__device__ __forceinline__ uint32_t float_key_of_bits(uint32_t u) {
  return u ^ ((u >> 31) ? 0xFFFFFFFFu : 0x80000000u);
}

// stream_keys for float input with a raw-bit test (run_to_raw): a key is
// formed only for the values that pass, as the queue hands them out; the
// queue's leftovers are turned into keys at the end, so the caller sees keys.
template <typename Src, typename Test, typename Take>
__device__ __forceinline__ void stream_raw_f32(Src& src, uint32_t* wq, uint32_t& qn, uint32_t lane, Test& test,
                                               Take&& take) {
  src.run([&](const uint4& qv) {
    const uint32_t e[4] = {qv.x, qv.y, qv.z, qv.w};
    bool hh[4];
    bool any = false;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      hh[t] = test(e[t]);
      any = any || hh[t];
    }
    if (!__any_sync(FULL, any)) return;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      uint32_t r0;
      if (wq_push(wq, qn, hh[t], e[t], lane, &r0)) take(float_key_of_bits(r0));
    }
  });
  __syncwarp();
  if (lane < qn) wq[lane] = float_key_of_bits(wq[lane]);
  __syncwarp();
}

// PASS 1 over windows with R runs (compile-time): the run tests, the per-run
// counts (CNT) into below[0..R), the keys inside a run to take().
template <typename T, uint32_t R, bool CNT, typename Src, typename Take>
__device__ __forceinline__ void count_runs(const Windows<typename KeyOf<T>::K>& W, Src& src,
                                           typename KeyOf<T>::K* wq, uint32_t& qn, uint32_t lane,
                                           uint32_t (&below)[L0_WIN], Take&& take) {
  using K = typename KeyOf<T>::K;
  if constexpr (std::is_same<T, float>::value && !CNT) {
    RunTest<K, R, false> tr;
    bool raw = true;
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) raw = raw && run_to_raw(W.lo[r], (K)(W.hi[r] - W.lo[r]), tr.lo[r], tr.sp[r]);
    if (raw) {  // the same for every thread (W is the CTA's copy)
      stream_raw_f32(src, wq, qn, lane, tr, take);
      return;
    }
  }
  RunTest<K, R, CNT> t;
#pragma unroll
  for (uint32_t r = 0; r < R; ++r) {
    t.lo[r] = W.lo[r];
    t.sp[r] = (K)(W.hi[r] - W.lo[r]);
    t.bl[r] = 0u;
  }
  stream_keys<T>(src, wq, qn, lane, t, take);
#pragma unroll
  for (uint32_t r = 0; r < R; ++r) below[r] = t.bl[r];
}

// PASS 1.  Persistent CTAs; each keeps a shared histogram of the B buckets.
// At the end a CTA adds its non-zero bins to the global histogram and writes
// its whole row to crow[blockIdx][*] -- PASS 2 turns those rows into private
// per-CTA write cursors, so it needs no global atomics.  Element -> CTA
// assignment is a pure function of (n, grid, NT, UNROLL, input alignment), the
// same in both passes.
// With windows (Windows::on) only the keys inside a run are bucketed (through
// the per-warp queue); every key bumps, per run r, a register count of the
// keys below the run's first key.  At the end the CTA's count of every gap
// follows -- gap g = below(run g) - below(run g-1) - count(run g-1), the last
// gap = all - below(last run) - count(last run) -- and goes to the gap's first
// bucket, so the prefix sums over the buckets stay exact.
template <typename T, int NT, int UNROLL>
__global__ __launch_bounds__(NT, PASS_MIN_CTAS(NT)) void l0_count(const T* __restrict__ in, uint64_t n,
                                              const Grid<typename KeyOf<T>::K>* __restrict__ Gs,
                                              Counters* C,
                                              const Windows<typename KeyOf<T>::K>* __restrict__ Wg,
                                              uint32_t* __restrict__ hist0, uint32_t* __restrict__ crow,
                                              uint32_t ring_st) {
  // the grid (final since the assigner, two or more kernels back) is loaded
  // while the predecessor, which zeroes hist0 and possibly the windows, ends
  pdl_trigger();
  using K = typename KeyOf<T>::K;
  constexpr int EPV = Vec16<T>::N;
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ Windows<K> W;
  __shared__ uint32_t red[NT / 32][2 * L0_WIN + 1];
  __shared__ RingBars rbars;
  const Grid<K>* G = Gs + C->asg_choice;
  uint2* s1 = (uint2*)smem;
  uint2* s2 = s1 + GRID_T1;
  uint32_t* hs = (uint32_t*)(smem + GRID_SMEM);
  GGMS_TRACE(24);
  GGMS_TRACE_CTA(0);
  const GridView<K> gv = grid_to_smem<K>(G, s1, s2);
  const uint32_t B = gv.B;
  K* wq = reinterpret_cast<K*>(hs + B) + (threadIdx.x >> 5) * WQ_DEPTH;
  for (uint32_t i = threadIdx.x; i < B; i += NT) hs[i] = 0u;
  pdl_wait();
  if (threadIdx.x == 0) W = *Wg;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&C->passes, 1u);
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;

  const uint64_t gtid = (uint64_t)blockIdx.x * NT + threadIdx.x;
  const uint64_t gstride = (uint64_t)gridDim.x * NT;
  uint64_t head = ((16u - (uint32_t)((uintptr_t)in & 15u)) & 15u) / sizeof(T);
  if (head > n) head = n;
  const uint64_t nvec = (n - head) / EPV;
  PassStream<NT, UNROLL> src;
  src.start(reinterpret_cast<const uint4*>(in + head), nvec,
            ring_at(smem, GRID_SMEM + (size_t)B * 4u + wq_bytes((uint32_t)NT, sizeof(K))), &rbars, ring_st);

  auto bucket = [&](K key) { return min(grid_eval<K>(gv, key), B - 1u); };
  // windows: this thread's count of keys below each run's first key (only
  // kept when two or more gaps hold keys, W.cnt)
  uint32_t below[L0_WIN] = {0u, 0u, 0u, 0u};
  uint32_t seen = 0;  // keys this thread counted (windows only)

  if (!W.on) {
    src.run([&](const uint4& qv) {
      T e[EPV];
      unpack16<T>(qv, e);
      uint32_t b[EPV];
#pragma unroll
      for (int t = 0; t < EPV; ++t) b[t] = bucket(KeyOf<T>::to(e[t]));
      bool same = true;
#pragma unroll
      for (int t = 1; t < EPV; ++t) same = same && (b[t] == b[0]);
      if (same) {
        atomicAdd(&hs[b[0]], (uint32_t)EPV);
      } else {
#pragma unroll
        for (int t = 0; t < EPV; ++t) atomicAdd(&hs[b[t]], 1u);
      }
    });
  } else {
    // R runs and (CNT) the per-run counts are compile-time, so that the bounds
    // and counts stay in registers
    uint32_t qn = 0;  // warp-uniform queue fill
    auto take = [&](K k) { atomicAdd(&hs[bucket(k)], 1u); };
    switch (W.R * 2u + (W.cnt ? 1u : 0u)) {
      case 2: count_runs<T, 1, false>(W, src, wq, qn, lane, below, take); break;
      case 3: count_runs<T, 1, true>(W, src, wq, qn, lane, below, take); break;
      case 4: count_runs<T, 2, false>(W, src, wq, qn, lane, below, take); break;
      case 5: count_runs<T, 2, true>(W, src, wq, qn, lane, below, take); break;
      case 6: count_runs<T, 3, false>(W, src, wq, qn, lane, below, take); break;
      case 7: count_runs<T, 3, true>(W, src, wq, qn, lane, below, take); break;
      case 8: count_runs<T, 4, false>(W, src, wq, qn, lane, below, take); break;
      default: count_runs<T, 4, true>(W, src, wq, qn, lane, below, take); break;
    }
    seen += (uint32_t)(src.my_vecs() * EPV);
    __syncwarp();
    if (lane < qn) atomicAdd(&hs[bucket(wq[lane])], 1u);
  }
  src.finish(C);
  // the partial last round, then the unaligned head and the tail that does not fill a vector
  auto tally = [&](K key) {
    if (!W.on) {
      atomicAdd(&hs[bucket(key)], 1u);
      return;
    }
    ++seen;
    bool h = false;
#pragma unroll
    for (uint32_t r = 0; r < L0_WIN; ++r) {
      if (r < W.R) {
        below[r] += key < W.lo[r] ? 1u : 0u;
        h = h | ((K)(key - W.lo[r]) <= (K)(W.hi[r] - W.lo[r]));
      }
    }
    if (h) atomicAdd(&hs[bucket(key)], 1u);
  };
  const T* vbase = in + head;
  for (uint64_t i = src.main_end + gtid; i < nvec; i += gstride) {
    T e[EPV];
    unpack16<T>(ld_stream16(vbase + i * EPV), e);
#pragma unroll
    for (int t = 0; t < EPV; ++t) tally(KeyOf<T>::to(e[t]));
  }
  {
    const uint64_t tail0 = head + nvec * EPV;
    const uint64_t nscalar = head + (n - tail0);
    for (uint64_t j = gtid; j < nscalar; j += gstride) {
      const uint64_t idx = j < head ? j : tail0 + (j - head);
      tally(KeyOf<T>::to(in[idx]));
    }
  }
  __syncthreads();
  if (W.on) {
    // this CTA's gap counts into the gaps' first buckets; red[w][*] holds warp
    // w's sums of: below(run r) for r < L0_WIN, count(run r), keys seen
#pragma unroll
    for (uint32_t r = 0; r < L0_WIN; ++r) {
      uint32_t hot = 0;
      if (r < W.R)
        for (uint32_t b = W.rb0[r] + threadIdx.x; b <= W.rb1[r]; b += NT) hot += hs[b];
      uint32_t x = below[r], y = hot;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(FULL, x, o);
        y += __shfl_xor_sync(FULL, y, o);
      }
      if (lane == 0) {
        red[threadIdx.x >> 5][r] = x;
        red[threadIdx.x >> 5][L0_WIN + r] = y;
      }
    }
    uint32_t z = seen;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(FULL, z, o);
    if (lane == 0) red[threadIdx.x >> 5][2 * L0_WIN] = z;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t below[L0_WIN], hot[L0_WIN], all = 0;
      for (uint32_t r = 0; r < L0_WIN; ++r) below[r] = hot[r] = 0u;
      for (uint32_t w = 0; w < NT / 32; ++w) {
        for (uint32_t r = 0; r < L0_WIN; ++r) {
          below[r] += red[w][r];
          hot[r] += red[w][L0_WIN + r];
        }
        all += red[w][2 * L0_WIN];
      }
      const uint32_t R = W.R;
      uint32_t rest = all;
      for (uint32_t r = 0; r < R; ++r) rest -= hot[r];
      for (uint32_t g = 0; g <= R; ++g) {
        if (W.gb0[g] > W.gb1[g]) continue;  // empty gap
        uint32_t gap;
        if (!W.cnt) gap = rest;  // the only gap that holds keys
        else if (g == 0) gap = below[0];
        else if (g < R) gap = below[g] - below[g - 1] - hot[g - 1];
        else gap = all - below[R - 1] - hot[R - 1];
        if (gap) hs[W.gb0[g]] += gap;
      }
    }
    __syncthreads();
  }
  uint32_t* row = crow + (size_t)blockIdx.x * B;
  for (uint32_t i = threadIdx.x; i < B; i += NT) {
    const uint32_t v = hs[i];
    row[i] = v;
    if (v) atomicAdd(&hist0[i], v);
  }
  GGMS_TRACE(25);
  GGMS_TRACE_CTA(1);
}

// Inclusive scan of the level-0 counts (one CTA) + the largest bucket.  The
// counts are staged through shared memory with coalesced loads/stores.
// With windows the gap buckets are left out of the largest-bucket statistic
// (a gap bucket counts a whole gap, not a bucket).
template <typename K>
__global__ __launch_bounds__(1024) void l0_scan(uint32_t* hist0, uint32_t B, Counters* C,
                                                const Windows<K>* __restrict__ Wg, uint32_t* aflagc) {
  pdl_entry();
  extern __shared__ uint32_t sh_counts[];
  __shared__ uint32_t w[72];
  __shared__ uint32_t mx;
  __shared__ Windows<K> W;
  GGMS_TRACE(26);
  if (threadIdx.x == 0) {
    W = *Wg;
    mx = 0;
  }
  if (threadIdx.x < NGRP / 32) aflagc[threadIdx.x] = 0u;  // the coarse mode's group flags
  __syncthreads();
  const bool on = W.on != 0u;
  uint32_t m = 0;
  for (uint32_t i = threadIdx.x; i < B; i += 1024) {
    const uint32_t v = hist0[i];
    sh_counts[i] = v;
    if (on) {
      bool gap = false;
#pragma unroll
      for (uint32_t g = 0; g <= L0_WIN; ++g) gap = gap || (g <= W.R && i == W.gb0[g]);
      if (!gap) m = max(m, v);
    }
  }
  __syncthreads();
  if (on) atomicMax(&mx, m);
  block_inclusive_scan_global<1024>(sh_counts, B, w, &C->max_bucket0);
  for (uint32_t i = threadIdx.x; i < B; i += 1024) hist0[i] = sh_counts[i];
  if (on && threadIdx.x == 0) C->max_bucket0 = mx;
  GGMS_TRACE(27);
}

// Each k finds the bucket holding its rank: the smallest b with I[b] > r
// (I: the inclusive counts of its segment's row).  Returns the bucket, or
// K_NIL when the rank lies beyond the row (cannot happen; status set).
__device__ __forceinline__ uint32_t locate_one(const uint32_t* I, uint32_t row_len, uint32_t& r, Counters* C) {
  if (r >= I[row_len - 1]) {  // cannot happen: rank beyond the segment
    set_status(C, GGMS_E_INTERNAL);
    return K_NIL;
  }
  uint32_t lo = 0, hi = row_len - 1;
  while (lo < hi) {
    const uint32_t m = (lo + hi) >> 1;
    if (I[m] > r) hi = m; else lo = m + 1;
  }
  r -= lo ? I[lo - 1] : 0u;
  return lo;
}

// With kcnt (level 0 of one vector), the ks of each bucket are also counted.
__global__ void lvl_locate_rows(const uint32_t* __restrict__ rows, uint32_t row_len, uint32_t nk,
                                uint32_t* k_rank, const uint32_t* __restrict__ k_seg,
                                uint32_t* k_bin, uint32_t* aflag, uint32_t flag_words,
                                Counters* C, uint32_t* kcnt = nullptr) {
  pdl_entry();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nk) return;
  const uint32_t s = k_seg[i];
  if (s == K_DONE) return;
  uint32_t r = k_rank[i];
  const uint32_t lo = locate_one(rows + (size_t)s * row_len, row_len, r, C);
  if (lo == K_NIL) return;
  k_bin[i] = lo;
  k_rank[i] = r;
  atomicOr(&aflag[(size_t)s * flag_words + (lo >> 5)], 1u << (lo & 31));
  if (kcnt) atomicAdd(&kcnt[lo], 1u);
}

// Active level-0 buckets -> refinement segments (or points).  In the coarse
// mode (C->coarse) the children are the NGRP groups of 2^gsh consecutive
// buckets instead (counts from ic, flags from aflagc).  A child of at most
// tiny_keys keys that holds at most TS_SORT_ABOVE ks (kcnt0) is finished by
// one warp (tiny_select), a larger small one by one CTA.
constexpr uint32_t TS_SORT_ABOVE = 8;

// Level-0 children: one thread per bucket (or, coarse, per group) holding a k.
// A child is a point (a single key: answered from `points`) or a segment with
// its key range [L(b), L(b+1) - 1], L(x) = smallest key with bucket >= x (a gap
// bucket of the windows stands for its whole gap; a group for its buckets),
// finished by the warp or CTA selects or refined by a level.  Ids in the
// shared lists are reserved per block: shared atomics inside the block, then
// one global atomic per counter -- a global counter bumped by every active
// bucket serialises ~10^3 same-address atomics in L2.
template <typename K>
__global__ __launch_bounds__(1024) void l0_children(const uint32_t* __restrict__ I,
                                                    const uint32_t* __restrict__ aflag,
                            uint32_t B, const Grid<K>* __restrict__ Gs, Counters* C,
                            const Windows<K>* __restrict__ Wg,
                            uint32_t* cmap0, Seg<K>* segs1, uint32_t* cursor1, TileRef* tiles1,
                            K* points, uint32_t* khead1, uint32_t* smalls, uint32_t* bigs1, Caps caps,
                            const uint32_t* __restrict__ ic, const uint32_t* __restrict__ aflagc,
                            const uint32_t* __restrict__ kcnt0, uint32_t tiny_keys, uint32_t* tinies) {
  pdl_trigger();  // the grid is loaded before the wait (it is older than the predecessor's output)
  // the key-range searches read the grid a few dozen times per bucket: keep
  // it in shared memory (every thread helps load it before any returns)
  __shared__ uint2 s1[GRID_T1];
  __shared__ uint2 s2[GRID_SUBCAP];
  enum { N_ACT, N_PT, N_SEG, N_TINY, N_SMALL, N_BIG, N_TILE, N_CTR };
  __shared__ uint32_t ctr[N_CTR], cbase[N_CTR];
  __shared__ unsigned long long cand_s;
  if (threadIdx.x < N_CTR) ctr[threadIdx.x] = 0u;
  if (threadIdx.x == 0) cand_s = 0ull;
  GGMS_TRACE(28);
  const Grid<K>* G = Gs + C->asg_choice;
  const GridView<K> gv = grid_to_smem<K>(G, s1, s2);
  const uint32_t ncell = G->ncell;
  pdl_wait();
  __syncthreads();
  GGMS_TRACE(29);
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  const bool coarse = C->coarse != 0u;
  const uint32_t gsh = coarse_shift(B);
  const uint32_t* Ib = coarse ? ic : I;
  // 1. classify this thread's bucket and take its block-local slots
  enum { C_NONE, C_POINT, C_TINY, C_SMALL, C_BIG };
  uint32_t kind = C_NONE, start = 0, cnt = 0, li = 0, lt = 0, nt = 0, ls = 0;
  K lo = 0, hi = 0;
  if (b < (coarse ? NGRP : B)) {
    if (!(((coarse ? aflagc : aflag)[b >> 5] >> (b & 31)) & 1u)) {
      cmap0[b] = CM_NONE;
    } else {
      start = b ? Ib[b - 1] : 0u;
      cnt = Ib[b] - start;
      const uint32_t b0 = coarse ? b << gsh : b;
      const uint32_t e = coarse ? ((b + 1u) << gsh) - 1u : win_end<K>(*Wg, b);
      lo = (b0 == 0) ? (K)0 : grid_inv<K>(gv, ncell, b0);
      hi = grid_last_key<K>(gv, ncell, e);
      atomicAdd(&ctr[N_ACT], 1u);
      if (lo == hi) {
        kind = C_POINT;
        li = atomicAdd(&ctr[N_PT], 1u);
      } else {
        ls = atomicAdd(&ctr[N_SEG], 1u);
        atomicAdd(&cand_s, (unsigned long long)cnt);
        if (cnt <= caps.small_keys) {
          kind = (!coarse && cnt <= tiny_keys && kcnt0[b] <= TS_SORT_ABOVE) ? C_TINY : C_SMALL;
          li = atomicAdd(&ctr[kind == C_TINY ? N_TINY : N_SMALL], 1u);
        } else {
          kind = C_BIG;
          li = atomicAdd(&ctr[N_BIG], 1u);
          nt = (cnt + TILE - 1) / TILE;
          lt = atomicAdd(&ctr[N_TILE], nt);
        }
      }
    }
  }
  __syncthreads();
  GGMS_TRACE(58);
  // 2. the block's ranges in the shared lists: one lane per counter, so the
  //    global atomics (each an L2 round trip) are in flight together
  if (threadIdx.x < 32u && ctr[N_ACT]) {
    const uint32_t t = threadIdx.x;
    uint32_t* const cp = t == N_ACT ? &C->active0 : t == N_PT ? &C->npoints : t == N_SEG ? &C->nsegs[1]
                         : t == N_TINY ? &C->ntiny : t == N_SMALL ? &C->nsmall : t == N_BIG ? &C->nbig[1]
                                                                                            : &C->ntiles[1];
    if (t < N_CTR && ctr[t]) cbase[t] = atomicAdd(cp, ctr[t]);
    if (t == N_CTR && ctr[N_PT]) atomicAdd(&C->point0, ctr[N_PT]);
    if (t == N_CTR + 1u && ctr[N_SEG]) atomicAdd(&C->cand0, cand_s);
  }
  __syncthreads();
  GGMS_TRACE(59);
  // 3. write this thread's child
  if (kind == C_NONE) return;
  if (kind == C_POINT) {
    const uint32_t pid = cbase[N_PT] + li;
    if (pid >= caps.points) { set_status(C, GGMS_E_INTERNAL); cmap0[b] = CM_NONE; return; }
    points[pid] = lo;
    cmap0[b] = CM_POINT | pid;
    return;
  }
  const uint32_t id = cbase[N_SEG] + ls;
  if (id >= caps.segs) { set_status(C, GGMS_E_INTERNAL); cmap0[b] = CM_NONE; return; }
  Seg<K> sg;
  sg.off = start;
  sg.cnt = cnt;
  sg.lo = lo;
  sg.hi = hi;
  sg.shift = (uint32_t)max(0, bitlen((K)(hi - lo)) - RADIX_BITS);
  sg.small = kind != C_BIG ? 1u : 0u;
  sg.pad = b;  // the level-0 bucket or group (l0_bases needs it)
  segs1[id] = sg;
  cursor1[id] = 0u;
  khead1[id] = K_NIL;
  cmap0[b] = id;
  if (kind != C_BIG) {
    const uint32_t si = cbase[kind == C_TINY ? N_TINY : N_SMALL] + li;
    if (si < caps.segs) (kind == C_TINY ? tinies : smalls)[si] = id; else set_status(C, GGMS_E_INTERNAL);
    return;
  }
  const uint32_t bi = cbase[N_BIG] + li;
  if (bi < caps.segs) bigs1[bi] = id; else set_status(C, GGMS_E_INTERNAL);
  const uint32_t t0 = cbase[N_TILE] + lt;
  if (t0 + nt > caps.tiles || t0 + nt < t0) { set_status(C, GGMS_E_INTERNAL); return; }
  for (uint32_t t = 0; t < nt; ++t) tiles1[t0 + t] = TileRef{id, t};
}

// ks follow their bin: resolved (single key) or the id of the next segment.
template <typename K>
__device__ __forceinline__ void relabel_one(uint32_t i, uint32_t e, uint32_t* k_seg, K* k_key,
                                            const K* __restrict__ points, Counters* C,
                                            const Seg<K>* __restrict__ segs_q, uint32_t* khead_q,
                                            uint32_t* knext) {
  if (e == CM_NONE) {
    set_status(C, GGMS_E_INTERNAL);
    k_seg[i] = K_DONE;
    return;
  }
  if (e & CM_POINT) {
    k_key[i] = points[e & ~CM_POINT];
    k_seg[i] = K_DONE;
  } else {
    k_seg[i] = e;
    if (segs_q[e].small) knext[i] = atomicExch(&khead_q[e], i);  // lock-free push
  }
}

template <typename K>
__global__ void lvl_relabel(const uint32_t* __restrict__ cmap, uint32_t row_len, uint32_t nk,
                            const uint32_t* __restrict__ k_bin, uint32_t* k_seg, K* k_key,
                            const K* __restrict__ points, Counters* C,
                            const Seg<K>* __restrict__ segs_q, uint32_t* khead_q, uint32_t* knext) {
  pdl_entry();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nk) return;
  const uint32_t s = k_seg[i];
  if (s == K_DONE) return;
  relabel_one<K>(i, cmap[(size_t)s * row_len + k_bin[i]], k_seg, k_key, points, C, segs_q, khead_q, knext);
}

// The first steps between PASS 1 and PASS 2 of one vector in ONE CTA (1024
// threads), through shared memory: the scan of the bucket counts, every k's
// bucket and rank in it, and the coarse-mode decision with the groups' counts
// and flags -- what l0_scan, lvl_locate_rows and l0_mode_ks do in three
// launches.  l0_children and l0_relabel_bases follow.  Dynamic shared memory:
// l0_between_smem(B).
__host__ __device__ constexpr size_t l0_between_smem(uint32_t B) {
  return 4u * (size_t)B + 4u * ((size_t)B / 32u);
}

template <typename K>
__global__ __launch_bounds__(1024) void l0_between(uint32_t* hist0, uint32_t B, Counters* C,
                                                   const Windows<K>* __restrict__ Wg, uint32_t nk,
                                                   uint32_t* k_rank, const uint32_t* __restrict__ k_seg,
                                                   uint32_t* k_bin, uint32_t* kcnt0, uint32_t* aflag0,
                                                   uint32_t* ic, uint32_t* aflagc) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ Windows<K> W;
  __shared__ uint32_t red[72];
  __shared__ uint32_t mx, ntot;
  __shared__ uint32_t afc[NGRP / 32];
  GGMS_TRACE(26);
  uint32_t* I = reinterpret_cast<uint32_t*>(smem);  // [B] counts, then inclusive counts
  uint32_t* af = I + B;                             // [B / 32] buckets holding a k
  const uint32_t tid = threadIdx.x;
  if (tid == 0) {
    W = *Wg;
    mx = 0;
    ntot = 0;
  }
  if (tid < NGRP / 32) afc[tid] = 0u;
  for (uint32_t w = tid; w < B / 32; w += 1024) af[w] = 0u;
  __syncthreads();
  // 1. inclusive scan of the counts (and the largest bucket outside the gap buckets)
  const bool on = W.on != 0u;
  uint32_t m = 0;
  for (uint32_t i0 = tid; i0 < B; i0 += 8u * 1024u) {  // 8 loads in flight per thread
    uint32_t v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t i = i0 + (uint32_t)u * 1024u;
      v[u] = i < B ? hist0[i] : 0u;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t i = i0 + (uint32_t)u * 1024u;
      if (i >= B) break;
      I[i] = v[u];
      if (on) {
        bool gap = false;
#pragma unroll
        for (uint32_t g = 0; g <= L0_WIN; ++g) gap = gap || (g <= W.R && i == W.gb0[g]);
        if (!gap) m = max(m, v[u]);
      }
    }
  }
  __syncthreads();
  if (on) atomicMax(&mx, m);
  block_inclusive_scan_global<1024>(I, B, red, &C->max_bucket0);
  for (uint32_t i = tid; i < B; i += 1024) hist0[i] = I[i];
  if (on && tid == 0) C->max_bucket0 = mx;
  GGMS_TRACE(43);
  // 2. every k: its bucket and its rank inside it
  for (uint32_t i = tid; i < nk; i += 1024) {
    if (k_seg[i] == K_DONE) continue;
    uint32_t r = k_rank[i];
    const uint32_t b = locate_one(I, B, r, C);
    if (b == K_NIL) continue;
    k_bin[i] = b;
    k_rank[i] = r;
    atomicOr(&af[b >> 5], 1u << (b & 31));
    atomicAdd(&kcnt0[b], 1u);
  }
  __syncthreads();
  GGMS_TRACE(44);
  // 3. coarse mode: most buckets hold a k (and no windows): groups of buckets
  uint32_t a = 0;
  for (uint32_t w = tid; w < B / 32; w += 1024) {
    const uint32_t f = af[w];
    aflag0[w] = f;
    a += __popc(f);
  }
  atomicAdd(&ntot, a);
  const uint32_t gsh = coarse_shift(B);
  for (uint32_t g = tid; g < NGRP; g += 1024) ic[g] = I[((g + 1u) << gsh) - 1u];
  __syncthreads();
  const bool coarse = !on && ntot * 2u >= B;
  if (tid == 0) C->coarse = coarse ? 1u : 0u;
  if (coarse) {
    for (uint32_t i = tid; i < nk; i += 1024) {
      if (k_seg[i] == K_DONE) continue;
      const uint32_t b = k_bin[i], g = b >> gsh, g0 = g << gsh;
      k_rank[i] += (b ? I[b - 1] : 0u) - (g0 ? I[g0 - 1] : 0u);
      k_bin[i] = g;
      atomicOr(&afc[g >> 5], 1u << (g & 31));
    }
  }
  __syncthreads();
  if (tid < NGRP / 32) aflagc[tid] = afc[tid];
  GGMS_TRACE(45);
}

// Per-CTA write cursors for PASS 2: for every level-0 child (a copied bucket
// b), one warp turns column b of the per-CTA count rows into exclusive
// prefixes plus the child's offset, in place.  CTA g of PASS 2 then owns the
// slots [crow[g][b], crow[g][b] + its count) of bucket b.
template <typename K>
__device__ __forceinline__ void bases_body(uint32_t* crow, uint32_t B, uint32_t ncta, const Seg<K>* __restrict__ segs1,
                                           const Counters* __restrict__ C, const Caps& caps) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  GGMS_TRACE(30);
  const uint32_t ns = min(C->nsegs[1], caps.segs);
  const bool coarse = C->coarse != 0u;
  const uint32_t gsh = coarse_shift(B);
  for (uint32_t id = warp; id < ns; id += (gridDim.x * blockDim.x) >> 5) {
    const Seg<K> s = segs1[id];
    // the level-0 bucket this child came from (coarse: the first bucket of its
    // group, whose column then holds the group's cursors)
    const uint32_t b = coarse ? s.pad << gsh : s.pad;
    uint64_t run = s.off;
    // a column of up to 256 CTAs' counts per batch, all loads in flight at once
    constexpr int BB = 8;
    for (uint32_t g0 = 0; g0 < ncta; g0 += 32u * BB) {
      uint32_t v[BB];
#pragma unroll
      for (int u = 0; u < BB; ++u) {
        const uint32_t g = g0 + (uint32_t)u * 32u + lane;
        v[u] = 0u;
        if (g < ncta) {
          if (coarse)
            for (uint32_t j = 0; j < (1u << gsh); ++j) v[u] += crow[(size_t)g * B + b + j];
          else
            v[u] = crow[(size_t)g * B + b];
        }
      }
#pragma unroll
      for (int u = 0; u < BB; ++u) {
        const uint32_t g = g0 + (uint32_t)u * 32u + lane;
        uint32_t inc = v[u];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(FULL, inc, o);
          if ((int)lane >= o) inc += t;
        }
        if (g < ncta) crow[(size_t)g * B + b] = (uint32_t)(run + inc - v[u]);
        run += __shfl_sync(FULL, inc, 31);
      }
    }
  }
}

template <typename K>
__global__ void l0_bases(uint32_t* crow, uint32_t B, uint32_t ncta, const Seg<K>* __restrict__ segs1,
                         const Counters* __restrict__ C, Caps caps) {
  pdl_entry();
  bases_body<K>(crow, B, ncta, segs1, C, caps);
}

// After l0_children: the ks follow their level-0 child (lvl_relabel) and the
// per-CTA write cursors of PASS 2 are formed (l0_bases), in one launch --
// threads [0, nk) relabel, all warps then take children for the cursors.
// In a captured graph it also sets the condition of the first refinement
// level (lev1, nonzero): whether some level-0 child needs one.
template <typename K>
__global__ void l0_relabel_bases(const uint32_t* __restrict__ cmap0, uint32_t nk,
                                 const uint32_t* __restrict__ k_bin, uint32_t* k_seg, K* k_key,
                                 const K* __restrict__ points, Counters* C, const Seg<K>* __restrict__ segs1,
                                 uint32_t* khead1, uint32_t* knext, uint32_t* crow, uint32_t B, uint32_t ncta,
                                 Caps caps, cudaGraphConditionalHandle lev1) {
  pdl_entry();
  GGMS_TRACE(60);
  if (lev1 && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(lev1, C->nbig[1] ? 1u : 0u);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += gridDim.x * blockDim.x) {
    const uint32_t s = k_seg[i];
    if (s == K_DONE) continue;
    relabel_one<K>(i, cmap0[k_bin[i]], k_seg, k_key, points, C, segs1, khead1, knext);
  }
  GGMS_TRACE(61);
  bases_body<K>(crow, B, ncta, segs1, C, caps);
}

// PASS 2.  Re-reads the input with the same element -> CTA assignment as
// PASS 1; a key whose bucket is copied goes to slot atomicAdd(&cur[b], 1) of
// this CTA's private range (a shared-memory atomic: no global round trip).
// A shared bitmask says which buckets are copied (not points, not inactive).
// Most keys lie in grid cells without a copied bucket: a second bitmask over
// the grid's top-level cells ("hot" cells) rejects those with one shift and
// one shared load, before the bucket is computed.
// Keys that pass the cell test go through the per-warp queue (wq_push).
constexpr uint32_t MAX_B0 = 1u << 15;
constexpr uint32_t HOT_WORDS = (GRID_T1 + 31) / 32;
constexpr uint32_t L0_RUNS = 4;    // hot-cell runs tested by key compares (more: the cell bitmask)

// 32-bit words of the region shared by the prologue's prefix table and,
// afterwards, the per-warp queues.
__host__ __device__ constexpr uint32_t l0_compact_qwords(uint32_t nt, uint32_t key_bytes) {
  return (MAX_B0 / 32 + 1) > (nt / 32) * WQ_DEPTH * key_bytes / 4 ? (MAX_B0 / 32 + 1)
                                                                   : (nt / 32) * WQ_DEPTH * key_bytes / 4;
}

template <typename T, int NT, int UNROLL>
__global__ __launch_bounds__(NT, PASS_MIN_CTAS(NT)) void l0_compact(const T* __restrict__ in, uint64_t n,
                                                const Grid<typename KeyOf<T>::K>* __restrict__ Gs,
                                                Counters* C,
                                                const Windows<typename KeyOf<T>::K>* __restrict__ Wg,
                                                const uint32_t* __restrict__ cmap0,
                                                const uint32_t* __restrict__ crow,
                                                typename KeyOf<T>::K* dst, uint64_t dst_cap,
                                                uint32_t ring_st, const uint32_t* __restrict__ I0) {
  // Before the wait: the grid, the windows, the child map and the counts (all
  // from two or more kernels back); after it: the write cursors (crow), which
  // the predecessor (l0_relabel_bases) forms.
  pdl_trigger();
  using K = typename KeyOf<T>::K;
  constexpr int EPV = Vec16<T>::N;
  if (C->coarse) {  // l0_compact_coarse copies this call's groups
    pdl_wait();
    return;
  }
  GGMS_TRACE(32);
  GGMS_TRACE_CTA(2);
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ Windows<K> W;
  __shared__ RingBars rbars;
  if (threadIdx.x == 0) W = *Wg;
  const Grid<K>* G = Gs + C->asg_choice;
  uint2* s1 = (uint2*)smem;
  uint2* s2 = s1 + GRID_T1;
  uint32_t* amask = (uint32_t*)(smem + GRID_SMEM);  // [MAX_B0 / 32]
  uint32_t* wpre = amask + MAX_B0 / 32;              // [MAX_B0 / 32 + 1]: copied buckets before word w
  constexpr uint32_t QW = l0_compact_qwords(NT, sizeof(K));
  uint32_t* hot = wpre + QW;                         // [HOT_WORDS]
  uint32_t* cur = hot + HOT_WORDS;                   // [B]
  const GridView<K> gv = grid_to_smem<K>(G, s1, s2);
  const uint32_t B = gv.B, ncell = G->ncell;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t* myrow = crow + (size_t)blockIdx.x * B;
  for (uint32_t w = warp; w < B / 32; w += NT / 32) {
    const uint32_t b = w * 32 + lane;
    const uint32_t bits = __ballot_sync(FULL, cmap0[b] < CM_POINT);
    if (lane == 0) {
      amask[w] = bits;
      wpre[w] = __popc(bits);
    }
  }
  // The cell bitmasks and runs below read only what kernels two or more back
  // wrote (the grid, windows, child map and counts), so they are built before
  // the dependency wait, while the write cursors are still being formed.
  __shared__ unsigned long long hot_mass_s;
  __shared__ K run_lo[L0_RUNS], run_span[L0_RUNS];
  __shared__ uint32_t nruns_s, ncopied_s;
  if (threadIdx.x == 0) {
    hot_mass_s = 0ull;
    nruns_s = 0u;
    ncopied_s = 0u;
  }
  __syncthreads();
  // With windows and no gap bucket to copy, every copied bucket lies inside a
  // window run: when the runs are narrow (tight), their key ranges (few, known
  // exactly) are the key test, and the hot cells below are not needed (every
  // thread decides the same from W and the mask).
  bool use_win = W.on != 0u && W.tight != 0u;
  for (uint32_t g = 0; g <= L0_WIN && use_win; ++g)
    if (g <= W.R && W.gb0[g] <= W.gb1[g] && ((amask[W.gb0[g] >> 5] >> (W.gb0[g] & 31)) & 1u))
      use_win = false;
  // with windows, a key outside every run belongs to its gap's bucket
  auto bmap = [&](uint32_t b) { return W.on ? win_map(W, b) : b; };
  if (use_win) {
    // the keys past the main part are tested by their bucket alone
    for (uint32_t w = threadIdx.x; w < HOT_WORDS; w += NT) hot[w] = FULL;
  } else {
    for (uint32_t w = threadIdx.x; w < HOT_WORDS; w += NT) hot[w] = 0u;
    if (warp == 0) {  // exclusive prefix of the per-word counts (B / 32 <= 1024 words)
      uint32_t run = 0;
      for (uint32_t w0 = 0; w0 < B / 32; w0 += 32) {
        const uint32_t v = wpre[w0 + lane];
        uint32_t inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(FULL, inc, o);
          if ((int)lane >= o) inc += t;
        }
        wpre[w0 + lane] = run + inc - v;
        run += __shfl_sync(FULL, inc, 31);
      }
      if (lane == 0) {
        wpre[B / 32] = run;
        ncopied_s = run;
      }
    }
    __syncthreads();
    {
      // a cell is hot when a copied bucket lies in [bucket of its first key,
      // bucket of its last key] (the grid and bmap are monotone in the key)
      auto rank = [&](uint32_t b) {  // copied buckets below b, b <= B
        const uint32_t w = b >> 5;
        return (b & 31) ? wpre[w] + __popc(amask[w] & ((1u << (b & 31)) - 1u)) : wpre[w];
      };
      const K dmax = (K)(gv.gmax - gv.origin);
      unsigned long long mass = 0;  // keys of this thread's hot cells (the buckets they span, from PASS 1)
      for (uint32_t c = threadIdx.x; c < ncell; c += NT) {
        const K d0 = (K)c << gv.sh1;
        const K d1 = (c + 1u < ncell) ? (K)(((K)(c + 1u) << gv.sh1) - 1u) : dmax;
        const uint32_t lo = bmap(min(grid_eval<K>(gv, (K)(gv.origin + d0)), B - 1u));
        const uint32_t hi = bmap(min(grid_eval<K>(gv, (K)(gv.origin + min(d1, dmax))), B - 1u));
        if (rank(hi + 1u) != rank(lo)) {
          atomicOr(&hot[c >> 5], 1u << (c & 31));
          mass += I0[hi] - (lo ? I0[lo - 1] : 0u);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mass += __shfl_xor_sync(FULL, mass, o);
      if (lane == 0 && mass) atomicAdd(&hot_mass_s, mass);  // buckets shared by two cells count twice
    }
    __syncthreads();
    // Maximal runs of hot cells as key intervals [lo, lo + span]; with at most
    // L0_RUNS of them the cell test becomes a few compares in registers.
    if (threadIdx.x == 0) {
      uint32_t nr = 0, start = 0;
      bool in_run = false;
      auto record = [&](uint32_t c0, uint32_t c1) {
        if (nr < L0_RUNS) {
          const K lo = (c0 == 0) ? (K)0 : (K)(gv.origin + ((K)c0 << gv.sh1));
          const K hi = (c1 + 1u >= ncell) ? key_max<K>() : (K)(gv.origin + ((K)(c1 + 1u) << gv.sh1) - 1u);
          run_lo[nr] = lo;
          run_span[nr] = (K)(hi - lo);
        }
        ++nr;
      };
      for (uint32_t w = 0; w < HOT_WORDS && nr <= L0_RUNS; ++w) {
        const uint32_t bits = hot[w];
        if ((!in_run && bits == 0u) || (in_run && bits == FULL)) continue;
        for (uint32_t b = 0; b < 32; ++b) {
          const uint32_t c = w * 32 + b;
          const bool hb = c < ncell && ((bits >> b) & 1u);
          if (hb && !in_run) {
            in_run = true;
            start = c;
          } else if (!hb && in_run) {
            in_run = false;
            record(start, c - 1u);
          }
        }
      }
      if (in_run) record(start, ncell - 1u);
      nruns_s = nr;
    }
  }
  pdl_wait();
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&C->passes, 1u);
  // the write cursors, 8 loads in flight per thread (this is on the critical path)
  for (uint32_t b0 = threadIdx.x; b0 < B; b0 += 8u * NT) {
    uint32_t v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t b = b0 + (uint32_t)u * NT;
      v[u] = (b < B && ((amask[b >> 5] >> (b & 31)) & 1u)) ? myrow[b] : 0u;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t b = b0 + (uint32_t)u * NT;
      if (b < B) cur[b] = v[u];
    }
  }
  __syncthreads();
  const uint32_t ncopied = ncopied_s;
  GGMS_TRACE(33);

  const uint64_t gtid = (uint64_t)blockIdx.x * NT + threadIdx.x;
  const uint64_t gstride = (uint64_t)gridDim.x * NT;
  uint64_t head = ((16u - (uint32_t)((uintptr_t)in & 15u)) & 15u) / sizeof(T);
  if (head > n) head = n;
  const uint64_t nvec = (n - head) / EPV;
  PassStream<NT, UNROLL> src;
  src.start(reinterpret_cast<const uint4*>(in + head), nvec,
            ring_at(smem, GRID_SMEM + (size_t)(MAX_B0 / 32 + QW + HOT_WORDS + B) * 4u), &rbars, ring_st);
  bool overflow = false;
  auto put = [&](uint32_t b, K key) {
    const uint32_t slot = atomicAdd(&cur[b], 1u);
    if (slot < dst_cap) dst[slot] = key; else overflow = true;
  };
  auto in_hot = [&](K key) {
    const K kc = min(max(key, gv.origin), gv.gmax);
    const uint32_t c = (uint32_t)((K)(kc - gv.origin) >> gv.sh1);
    return (hot[c >> 5] >> (c & 31)) & 1u;
  };

  auto bucket_and_put = [&](K key) {
    const uint32_t b = bmap(min(grid_eval<K>(gv, key), B - 1u));
    if ((amask[b >> 5] >> (b & 31)) & 1u) put(b, key);
  };
  // the per-warp queue lives where the prefix table was (dead after the prologue)
  K* wq = reinterpret_cast<K*>(wpre) + (threadIdx.x >> 5) * WQ_DEPTH;
  uint32_t qn = 0;  // warp-uniform

  // every lane runs the same number of rounds, so the warp stays converged
  const uint32_t nruns = nruns_s;
  auto runs = [&](auto rc, bool win) {
    constexpr uint32_t R = decltype(rc)::value;
    RunTest<K, R, false> t;
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) {
      t.lo[r] = win ? W.lo[r] : run_lo[r];
      t.sp[r] = win ? (K)(W.hi[r] - W.lo[r]) : run_span[r];
    }
    if constexpr (std::is_same<T, float>::value) {
      RunTest<K, R, false> tr;
      bool raw = true;
#pragma unroll
      for (uint32_t r = 0; r < R; ++r) raw = raw && run_to_raw(t.lo[r], t.sp[r], tr.lo[r], tr.sp[r]);
      if (raw) {  // the same for every thread of the CTA
        stream_raw_f32(src, wq, qn, lane, tr, bucket_and_put);
        return;
      }
    }
    stream_keys<T>(src, wq, qn, lane, t, bucket_and_put);
  };
  // Most buckets copied: every key takes the long path anyway, so the queue
  // only serialises it; each lane buckets its keys directly, all EPV of a
  // vector at once (independent lookups in flight).
  auto dense = [&]() {
    src.run([&](const uint4& qv) {
      T e[EPV];
      unpack16<T>(qv, e);
      K kk[EPV];
      uint32_t b[EPV];
#pragma unroll
      for (int t = 0; t < EPV; ++t) {
        kk[t] = KeyOf<T>::to(e[t]);
        b[t] = bmap(min(grid_eval<K>(gv, kk[t]), B - 1u));
      }
#pragma unroll
      for (int t = 0; t < EPV; ++t)
        if ((amask[b[t] >> 5] >> (b[t] & 31)) & 1u) put(b[t], kk[t]);
    });
  };
  // hot cells that hold most of the keys (ks spread over all ranks): every key
  // takes the long path anyway, so it goes there directly
  if (!use_win && nruns > L0_RUNS && (ncopied * 2u >= B || hot_mass_s * 2u > n)) {
    dense();
  } else if (use_win) {
    switch (W.R) {
      case 1: runs(std::integral_constant<uint32_t, 1>{}, true); break;
      case 2: runs(std::integral_constant<uint32_t, 2>{}, true); break;
      case 3: runs(std::integral_constant<uint32_t, 3>{}, true); break;
      default: runs(std::integral_constant<uint32_t, 4>{}, true); break;
    }
  } else switch (nruns) {
    case 0: break;  // nothing to copy
    case 1: runs(std::integral_constant<uint32_t, 1>{}, false); break;
    case 2: runs(std::integral_constant<uint32_t, 2>{}, false); break;
    case 3: runs(std::integral_constant<uint32_t, 3>{}, false); break;
    case 4: runs(std::integral_constant<uint32_t, 4>{}, false); break;
    default: stream_keys<T>(src, wq, qn, lane, in_hot, bucket_and_put); break;
  }
  src.finish(C);
  GGMS_TRACE(34);
  __syncwarp();
  if (lane < qn) bucket_and_put(wq[lane]);
  const T* vbase = in + head;
  for (uint64_t i = src.main_end + gtid; i < nvec; i += gstride) {
    T e[EPV];
    unpack16<T>(ld_stream16(vbase + i * EPV), e);
#pragma unroll
    for (int t = 0; t < EPV; ++t) {
      const K key = KeyOf<T>::to(e[t]);
      if (in_hot(key)) bucket_and_put(key);
    }
  }
  {
    const uint64_t tail0 = head + nvec * EPV;
    const uint64_t nscalar = head + (n - tail0);
    for (uint64_t j = gtid; j < nscalar; j += gstride) {
      const uint64_t idx = j < head ? j : tail0 + (j - head);
      const K key = KeyOf<T>::to(in[idx]);
      if (in_hot(key)) bucket_and_put(key);
    }
  }
  GGMS_TRACE_CTA(3);
  if (overflow) set_status(C, GGMS_E_INTERNAL);
}

// ------------------------------------------------------------------ coarse level 0
// When most buckets hold a k (many ks spread over all ranks), copying key by
// key into ~B per-CTA bucket ranges is a scatter of 4-byte stores over the
// whole candidate buffer, which runs far below the memory's bandwidth.  The
// coarse mode copies NGRP groups of consecutive buckets instead (equal mass,
// since the buckets are), and PASS 2 sorts each chunk of a CTA's keys by group
// in shared memory first, so that the stores leave as contiguous runs.  The
// refinement levels then split the groups.
// Decided on the device after PASS 1 (windows off and at least half the
// buckets flagged), by every CTA of l0_mode_ks for itself; CTA 0 records it
// and the groups' inclusive counts.  In the coarse mode a k's bucket becomes
// its group and its rank one inside the group.
template <typename K>
__global__ void l0_mode_ks(const uint32_t* __restrict__ I, const uint32_t* __restrict__ aflag0, uint32_t B,
                           const Windows<K>* __restrict__ Wg, Counters* C, uint32_t* ic, uint32_t* aflagc,
                           uint32_t nk, uint32_t* k_rank, const uint32_t* __restrict__ k_seg, uint32_t* k_bin) {
  pdl_entry();
  __shared__ uint32_t tot;
  GGMS_TRACE(38);
  if (threadIdx.x == 0) tot = 0u;
  __syncthreads();
  uint32_t a = 0;
  for (uint32_t w = threadIdx.x; w < B / 32; w += blockDim.x) a += __popc(aflag0[w]);
  atomicAdd(&tot, a);
  __syncthreads();
  const bool coarse = !Wg->on && tot * 2u >= B;
  const uint32_t gsh = coarse_shift(B);
  if (blockIdx.x == 0) {
    if (threadIdx.x == 0) C->coarse = coarse ? 1u : 0u;
    for (uint32_t g = threadIdx.x; g < NGRP; g += blockDim.x) ic[g] = I[((g + 1u) << gsh) - 1u];
  }
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (!coarse || i >= nk || k_seg[i] == K_DONE) return;
  const uint32_t b = k_bin[i], g = b >> gsh, g0 = g << gsh;
  k_rank[i] += (b ? I[b - 1] : 0u) - (g0 ? I[g0 - 1] : 0u);
  k_bin[i] = g;
  atomicOr(&aflagc[g >> 5], 1u << (g & 31));
}

// Keys of one PASS-2 chunk of the coarse mode: up to 4 vectors per thread.
// vectors per thread per staged chunk: up to 4 (the staged streams: 4)
__host__ __device__ constexpr int coarse_du(int unroll) { return unroll <= 0 ? 4 : (unroll < 4 ? unroll : 4); }
template <typename T, int NT, int UNROLL>
__host__ __device__ constexpr uint32_t coarse_chunk() {
  return (uint32_t)NT * coarse_du(UNROLL) * Vec16<T>::N;
}

// PASS 2 of the coarse mode.  Same element -> CTA assignment as PASS 1; CTA
// c's range of group g starts at crow[c][g << gsh] (l0_bases).  Per chunk: the
// group of every key (bucket >> gsh), its rank among the chunk's keys of that
// group (a shared atomic), a scan of the NGRP counts, the keys into shared
// memory in group order, then thread i stores staged key i -- consecutive
// threads, consecutive addresses inside a group's run.
template <typename T, int NT, int UNROLL>
__global__ __launch_bounds__(NT, PASS_MIN_CTAS(NT)) void l0_compact_coarse(const T* __restrict__ in, uint64_t n,
                                                       const Grid<typename KeyOf<T>::K>* __restrict__ Gs,
                                                       Counters* C, const uint32_t* __restrict__ cmap0,
                                                       const uint32_t* __restrict__ crow,
                                                       typename KeyOf<T>::K* dst, uint64_t dst_cap,
                                                       uint32_t ring_st) {
  pdl_entry();
  using K = typename KeyOf<T>::K;
  constexpr int EPV = Vec16<T>::N;
  constexpr int DU = coarse_du(UNROLL);
  constexpr uint32_t CH = coarse_chunk<T, NT, UNROLL>();
  constexpr uint32_t NONE = 0xFFFFFFFFu;
  static_assert(CH <= 65536u, "chunk ranks are 16-bit");
  if (!C->coarse) return;  // l0_compact copies this call's buckets
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&C->passes, 1u);
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint32_t gbase[NGRP], hist[NGRP], off[NGRP], cflag[NGRP / 32];
  __shared__ uint32_t total_s;
  __shared__ RingBars rbars;
  const Grid<K>* G = Gs + C->asg_choice;
  uint2* s1 = (uint2*)smem;
  uint2* s2 = s1 + GRID_T1;
  K* stg = (K*)(smem + GRID_SMEM);
  uint8_t* sg = (uint8_t*)(stg + CH);
  const GridView<K> gv = grid_to_smem<K>(G, s1, s2);
  const uint32_t B = gv.B, gsh = coarse_shift(B);
  const uint32_t tid = threadIdx.x, lane = tid & 31;
  if (tid < NGRP / 32) cflag[tid] = 0u;
  __syncthreads();
  for (uint32_t g = tid; g < NGRP; g += NT) {
    hist[g] = 0u;
    const bool copied = cmap0[g] < CM_POINT;
    gbase[g] = copied ? crow[(size_t)blockIdx.x * B + (g << gsh)] : 0u;
    if (copied) atomicOr(&cflag[g >> 5], 1u << (g & 31));
  }
  __syncthreads();
  auto group = [&](K key) -> uint32_t {
    const uint32_t g = min(grid_eval<K>(gv, key), B - 1u) >> gsh;
    return ((cflag[g >> 5] >> (g & 31)) & 1u) ? g : NONE;
  };

  const uint64_t gtid = (uint64_t)blockIdx.x * NT + tid;
  const uint64_t gstride = (uint64_t)gridDim.x * NT;
  uint64_t head = ((16u - (uint32_t)((uintptr_t)in & 15u)) & 15u) / sizeof(T);
  if (head > n) head = n;
  const uint64_t nvec = (n - head) / EPV;
  PassStream<NT, UNROLL> src;
  src.start(reinterpret_cast<const uint4*>(in + head), nvec,
            ring_at(smem, GRID_SMEM + (size_t)CH * (sizeof(K) + 1)), &rbars, ring_st);
  bool overflow = false;
  // One chunk: the first `got` of this thread's DU vectors (got is CTA-uniform).
  // The group of every key (bucket >> gsh), its rank among the chunk's keys of
  // that group (a shared atomic), a scan of the NGRP counts, the keys into
  // shared memory in group order, then thread i stores staged key i.
  auto stage = [&](const uint4 (&q)[DU], int got) {
    uint32_t pk[DU * EPV];  // (group << 16) | rank inside the chunk's group, or NONE
#pragma unroll
    for (int u = 0; u < DU; ++u) {
      T e[EPV];
      unpack16<T>(q[u], e);
      uint32_t g[EPV];
#pragma unroll
      for (int t = 0; t < EPV; ++t) g[t] = u < got ? group(KeyOf<T>::to(e[t])) : NONE;
#pragma unroll
      for (int t = 0; t < EPV; ++t)
        pk[u * EPV + t] = g[t] == NONE ? NONE : (g[t] << 16) | atomicAdd(&hist[g[t]], 1u);
    }
    __syncthreads();
    if (tid < 32) {  // exclusive scan of the NGRP counts, 8 per lane
      uint32_t c8[NGRP / 32], sum = 0;
#pragma unroll
      for (int j = 0; j < (int)(NGRP / 32); ++j) { c8[j] = hist[lane * (NGRP / 32) + j]; sum += c8[j]; }
      uint32_t inc = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, inc, o);
        if ((int)lane >= o) inc += t;
      }
      uint32_t run = inc - sum;
#pragma unroll
      for (int j = 0; j < (int)(NGRP / 32); ++j) { off[lane * (NGRP / 32) + j] = run; run += c8[j]; }
      if (lane == 31) total_s = inc;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < DU; ++u) {
      T e[EPV];
      unpack16<T>(q[u], e);
#pragma unroll
      for (int t = 0; t < EPV; ++t) {
        const uint32_t x = pk[u * EPV + t];
        if (x != NONE) {
          const uint32_t g = x >> 16, pos = off[g] + (x & 0xFFFFu);
          stg[pos] = KeyOf<T>::to(e[t]);
          sg[pos] = (uint8_t)g;
        }
      }
    }
    __syncthreads();
    const uint32_t tot = total_s;
    for (uint32_t i = tid; i < tot; i += NT) {
      const uint32_t g = sg[i];
      const uint64_t slot = (uint64_t)gbase[g] + (i - off[g]);
      if (slot < dst_cap) dst[slot] = stg[i]; else overflow = true;
    }
    __syncthreads();
    for (uint32_t g = tid; g < NGRP; g += NT) {
      gbase[g] += hist[g];
      hist[g] = 0u;
    }
    __syncthreads();
  };
  if constexpr (UNROLL > 0) {
    // chunk c: DU vectors of round c / CPR; the next chunk's loads are issued
    // before this chunk's barriers, so they are in flight while it is staged
    constexpr int CPR = UNROLL / DU;
    const uint4* vp = reinterpret_cast<const uint4*>(in + head) + gtid;
    const uint64_t nch = src.rounds * CPR;
    auto chunk_ptr = [&](uint64_t c) {
      return vp + (c / CPR) * gstride * UNROLL + (uint64_t)((int)(c % CPR) * DU) * gstride;
    };
    uint4 q[DU];
    if (nch) {
      const uint4* p0 = chunk_ptr(0);
#pragma unroll
      for (int u = 0; u < DU; ++u) q[u] = ld_stream16(p0 + u * gstride);
    }
    for (uint64_t c = 0; c < nch; ++c) {
      uint4 qn[DU];
      if (c + 1 < nch) {
        const uint4* pn = chunk_ptr(c + 1);
#pragma unroll
        for (int u = 0; u < DU; ++u) qn[u] = ld_stream16(pn + u * gstride);
      }
      stage(q, DU);
#pragma unroll
      for (int u = 0; u < DU; ++u) q[u] = qn[u];
    }
  } else {
    uint4 q[DU];
    for (int got; (got = src.template next_batch<DU>(q)) > 0;) stage(q, got);
  }
  src.finish(C);
  // the vectors past the main part, the unaligned head and the tail: one key at a time
  auto put = [&](K key) {
    const uint32_t g = group(key);
    if (g == NONE) return;
    const uint32_t slot = atomicAdd(&gbase[g], 1u);
    if (slot < dst_cap) dst[slot] = key; else overflow = true;
  };
  const T* vbase = in + head;
  for (uint64_t i = src.main_end + gtid; i < nvec; i += gstride) {
    T e[EPV];
    unpack16<T>(ld_stream16(vbase + i * EPV), e);
#pragma unroll
    for (int t = 0; t < EPV; ++t) put(KeyOf<T>::to(e[t]));
  }
  {
    const uint64_t tail0 = head + nvec * EPV;
    const uint64_t nscalar = head + (n - tail0);
    for (uint64_t j = gtid; j < nscalar; j += gstride) {
      const uint64_t idx = j < head ? j : tail0 + (j - head);
      put(KeyOf<T>::to(in[idx]));
    }
  }
  if (overflow) set_status(C, GGMS_E_INTERNAL);
}

// ------------------------------------------------------------------ refinement levels
// Level l works on the segments of pool p = l & 1 and creates children in pool
// q = p ^ 1.  Keys are read from `src` and children are written to `dst`.

// Gate of a refinement level inside a captured CUDA graph: the level (an IF
// node) runs only while every level so far had segments to refine.
__global__ void lvl_gate(Counters* C, int p, cudaGraphConditionalHandle h) {
  pdl_entry();
  GGMS_TRACE(41 + p);
  if (C->nbig[p] == 0u) C->done = 1u;
  cudaGraphSetConditional(h, C->done ? 0u : 1u);
}

// zero this level's histogram rows / flags (segments that small_select or
// tiny_select finished have none); reset the child pool's counters
__global__ void lvl_prep(uint32_t* rows, uint32_t* aflag, const uint32_t* __restrict__ bigs, Counters* C,
                         int p, Caps caps) {
  pdl_entry();
  const uint32_t nb = min(C->nbig[p], caps.segs);
  for (uint32_t j = blockIdx.x; j < nb; j += gridDim.x) {
    const uint32_t sid = bigs[j];
    uint32_t* row = rows + (size_t)sid * NBIN;
    for (uint32_t i = threadIdx.x; i < NBIN; i += blockDim.x) row[i] = 0u;
    for (uint32_t i = threadIdx.x; i < NBIN_WORDS; i += blockDim.x) aflag[(size_t)sid * NBIN_WORDS + i] = 0u;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    C->nsegs[p ^ 1] = 0u;
    C->ntiles[p ^ 1] = 0u;
    C->nbig[p ^ 1] = 0u;
    C->nsmall = 0u;
    C->ntiny = 0u;
    if (nb) C->levels_run += 1u;
  }
}

// Bin of a key in a quantile segment: the number of boundaries <= key.  The
// directory cell of the key bounds the search: boundaries before qd[c] lie
// below the cell's first key, those from qd[c + 1] on above its last.
template <typename K>
__device__ __forceinline__ uint32_t qbin(K key, K kmin, uint32_t dsh, const K* qb, const uint16_t* qd) {
  const K d = key > kmin ? (K)(key - kmin) : (K)0;
  const K cc = d >> dsh;
  const uint32_t c = cc < (K)QD ? (uint32_t)cc : QD - 1u;
  uint32_t lo = qd[c], hi = qd[c + 1];
  while (lo < hi) {
    const uint32_t m = (lo + hi) >> 1;
    if (qb[m] <= key) lo = m + 1; else hi = m;
  }
  return lo;
}

// Boundaries and directory of quantile segment q into shared memory.
template <typename K>
__device__ __forceinline__ void qtab_to_smem(const K* __restrict__ qtab, const uint16_t* __restrict__ qdir,
                                             uint32_t q, K* qb, uint16_t* qd) {
  const K* tb = qtab + (size_t)q * QB;
  for (uint32_t i = threadIdx.x; i < QB; i += blockDim.x) qb[i] = tb[i];
  const uint4* dr = reinterpret_cast<const uint4*>(qdir + (size_t)q * QDS);
  uint4* dd = reinterpret_cast<uint4*>(qd);
  for (uint32_t i = threadIdx.x; i < QDS / 8; i += blockDim.x) dd[i] = dr[i];
}

// Sample-quantile bins of the batched level 0: one CTA per large caller
// segment draws QSAMP keys (one from each of QSAMP equal strata, at a hashed
// offset inside it), sorts them, and writes the QB - 1 boundaries and the
// directory; the segment's lo / shift become the directory's origin / cell
// shift and pad its table index.
template <typename T>
__global__ __launch_bounds__(1024) void seg_sample(const T* __restrict__ in, Seg<typename KeyOf<T>::K>* segs0,
                                                   const uint32_t* __restrict__ qsegs,
                                                   const Counters* __restrict__ C, uint32_t cap_q,
                                                   typename KeyOf<T>::K* qtab, uint16_t* qdir, uint64_t seed) {
  pdl_entry();
  using K = typename KeyOf<T>::K;
  __shared__ K sv[QSAMP];
  const uint32_t tid = threadIdx.x;
  const uint32_t nq = min(C->nbig[0], cap_q);
  for (uint32_t q = blockIdx.x; q < nq; q += gridDim.x) {
    const uint32_t sid = qsegs[q];
    Seg<K> s = segs0[sid];
    for (uint32_t i = tid; i < QSAMP; i += 1024) {
      const uint64_t a = (uint64_t)s.cnt * i / QSAMP, b = (uint64_t)s.cnt * (i + 1) / QSAMP;
      const uint64_t h = mix64(seed ^ ((uint64_t)sid << 32) ^ i);
      const uint64_t pos = a + (((h >> 32) * (b - a)) >> 32);  // in [a, b) (b - a < 2^32), or a
      sv[i] = KeyOf<T>::to(in[s.off + pos]);
    }
    __syncthreads();
    for (uint32_t kk = 2; kk <= QSAMP; kk <<= 1) {
      for (uint32_t jj = kk >> 1; jj > 0; jj >>= 1) {
        for (uint32_t i = tid; i < QSAMP; i += 1024) {
          const uint32_t ixj = i ^ jj;
          if (ixj > i) {
            const K a = sv[i], b = sv[ixj];
            if ((a > b) == ((i & kk) == 0)) { sv[i] = b; sv[ixj] = a; }
          }
        }
        // stages with jj < 32 stay inside a warp (i and i ^ jj: lanes l, l ^ jj)
        const uint32_t nj = jj > 1 ? (jj >> 1) : kk;
        if (nj >= 32u || (jj == 1 && kk == QSAMP)) __syncthreads(); else __syncwarp();
      }
    }
    K* tb = qtab + (size_t)q * QB;
    for (uint32_t j = tid; j < QB; j += 1024) tb[j] = (j + 1 < QB) ? sv[2 * j + 2] : key_max<K>();
    const K kmin = sv[0], kmax = sv[QSAMP - 1];
    const uint32_t dsh = (uint32_t)max(0, bitlen((K)(kmax - kmin)) - QD_BITS);
    uint16_t* dr = qdir + (size_t)q * QDS;
    for (uint32_t c = tid; c < QDS; c += 1024) {
      uint32_t v = QB - 1u;  // past the range (or padding): every boundary is below
      const K off = (K)((K)c << dsh);
      if (c < QD && ((off >> dsh) == (K)c) && off <= (K)(key_max<K>() - kmin)) {
        const K start = (K)(kmin + off);
        uint32_t lo = 0, hi = QB - 1u;  // boundaries j < lo are < start
        while (lo < hi) {
          const uint32_t m = (lo + hi) >> 1;
          if (sv[2 * m + 2] < start) lo = m + 1; else hi = m;
        }
        v = lo;
      }
      dr[c] = (uint16_t)v;
    }
    if (tid == 0) {
      s.lo = kmin;
      s.shift = dsh;
      s.pad = q;
      segs0[sid] = s;
    }
    __syncthreads();
  }
}

// Histogram of radix bins, one tile of one segment per iteration.
// Q: the level's segments have quantile bins (batched level 0), else radix
// bins (key - lo) >> shift.
template <typename InT, int NT, bool Q = false>
__global__ __launch_bounds__(NT) void lvl_count(const InT* __restrict__ src,
                                               const Seg<typename KeyOf<InT>::K>* __restrict__ segs,
                                               const TileRef* __restrict__ tiles,
                                               Counters* C, int p, uint32_t* rows, Caps caps,
                                               const typename KeyOf<InT>::K* __restrict__ qtab,
                                               const uint16_t* __restrict__ qdir) {
  pdl_entry();
  using K = typename KeyOf<InT>::K;
  __shared__ uint32_t h[NBIN];
  __shared__ __align__(16) K qb[Q ? QB : 1];
  __shared__ __align__(16) uint16_t qd[Q ? QDS : 8];
  const uint32_t nt = min(C->ntiles[p], caps.tiles);
  const uint32_t ns = min(C->nsegs[p], caps.segs);
  if (Q && nt && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&C->passes, 1u);  // level 0 reads the input
  // Each CTA takes a contiguous range of the tile list, where a segment's tiles
  // are consecutive: the histogram of one segment's run of tiles stays in
  // shared memory and is added to the segment's row once per run, not once
  // per tile (a row holds NBIN bins for TILE keys), and the quantile table is
  // loaded once per run.
  const uint32_t per = (nt + gridDim.x - 1) / gridDim.x;
  const uint32_t t_beg = min(blockIdx.x * per, nt), t_end = min(t_beg + per, nt);
  uint32_t open = 0xFFFFFFFFu;  // segment whose counts the shared histogram holds
  unsigned long long open_keys = 0;
  auto flush = [&]() {  // all threads, after a barrier
    uint32_t* row = rows + (size_t)open * NBIN;
    for (uint32_t i = threadIdx.x; i < NBIN; i += NT) {
      const uint32_t v = h[i];
      if (v) atomicAdd(&row[i], v);
    }
    if (threadIdx.x == 0) atomicAdd(&C->refine_elems, open_keys);
  };
  for (uint32_t t = t_beg; t < t_end; ++t) {
    const TileRef tr = tiles[t];
    if (tr.seg >= ns) continue;  // only after a capacity error (status already set)
    const Seg<K> s = segs[tr.seg];
    if (tr.seg != open) {  // the previous tile ended with a barrier
      if (open != 0xFFFFFFFFu) {
        flush();
        __syncthreads();
      }
      if (Q) qtab_to_smem<K>(qtab, qdir, s.pad, qb, qd);
      for (uint32_t i = threadIdx.x; i < NBIN; i += NT) h[i] = 0u;
      open = tr.seg;
      open_keys = 0;
      __syncthreads();
    }
    const uint64_t beg = s.off + (uint64_t)tr.no * TILE;
    const uint64_t end = min(beg + TILE, s.off + s.cnt);
    constexpr int U = 8;  // independent loads in flight per thread
    for (uint64_t o = beg + threadIdx.x; o < end; o += (uint64_t)NT * U) {
      K kk[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint64_t i = o + (uint64_t)u * NT;
        kk[u] = i < end ? KeyOf<InT>::to(src[i]) : (K)0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (o + (uint64_t)u * NT >= end) break;
        uint32_t bin;
        if (Q) bin = qbin<K>(kk[u], s.lo, s.shift, qb, qd);
        else bin = min((uint32_t)((K)(kk[u] - s.lo) >> s.shift), (uint32_t)NBIN - 1u);
        atomicAdd(&h[bin], 1u);
      }
    }
    open_keys += end - beg;
    __syncthreads();
  }
  if (open != 0xFFFFFFFFu) flush();  // the last tile ended with a barrier
}

__global__ __launch_bounds__(1024) void lvl_scan(uint32_t* rows, const uint32_t* __restrict__ bigs,
                                                  const Counters* __restrict__ C, int p, Caps caps) {
  pdl_entry();
  __shared__ uint32_t w[72];
  const uint32_t nb = min(C->nbig[p], caps.segs);
  for (uint32_t j = blockIdx.x; j < nb; j += gridDim.x)
    block_inclusive_scan_global<1024>(rows + (size_t)bigs[j] * NBIN, NBIN, w, nullptr);
}

// Active bins of each segment -> child segments (pool q) or points.  One CTA
// per segment; the row holding the inclusive counts is overwritten by the
// child map (each entry read before any is written).
template <typename K, int NT, bool Q = false>
__global__ __launch_bounds__(NT) void lvl_children(uint32_t* rows, const uint32_t* __restrict__ aflag,
                                                  const Seg<K>* __restrict__ segs, Counters* C, int p,
                                                  Seg<K>* segs_q, uint32_t* cursor_q, TileRef* tiles_q,
                                                  K* points, uint32_t* khead_q, uint32_t* smalls,
                                                  uint32_t* tinies, const uint32_t* __restrict__ bigs,
                                                  uint32_t* bigs_q, Caps caps, const K* __restrict__ qtab) {
  pdl_entry();
  constexpr int PER = NBIN / NT;
  const uint32_t nb = min(C->nbig[p], caps.segs);
  for (uint32_t j = blockIdx.x; j < nb; j += gridDim.x) {
    const uint32_t sid = bigs[j];
    const Seg<K> s = segs[sid];
    if (s.small) continue;  // finished by small_select
    uint32_t* I = rows + (size_t)sid * NBIN;
    const uint32_t* F = aflag + (size_t)sid * NBIN_WORDS;
    uint32_t out[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const uint32_t b = threadIdx.x + u * NT;
      out[u] = CM_NONE;
      if (!((F[b >> 5] >> (b & 31)) & 1u)) continue;
      const uint32_t start = b ? I[b - 1] : 0u;
      const uint32_t cnt = I[b] - start;
      K blo, bhi;
      if (Q) {  // [boundary b - 1, boundary b - 1]; the outer bins reach the ends of the key space
        const K* tb = qtab + (size_t)s.pad * QB;
        blo = b ? tb[b - 1] : (K)0;
        bhi = (b + 1u < QB) ? (K)(tb[b] - 1u) : key_max<K>();
        if (b + 1u < QB && tb[b] <= blo) {  // an empty bin cannot hold a k
          set_status(C, GGMS_E_INTERNAL);
          continue;
        }
      } else {
        blo = s.lo + ((K)b << s.shift);
        const K width_m1 = (K)(((K)1 << s.shift) - 1);
        bhi = (key_max<K>() - blo < width_m1) ? key_max<K>() : (K)(blo + width_m1);
      }
      if (bhi > s.hi) bhi = s.hi;
      if (blo == bhi) {
        uint32_t pid = atomicAdd(&C->npoints, 1u);
        if (pid >= caps.points) { set_status(C, GGMS_E_INTERNAL); continue; }
        points[pid] = blo;
        out[u] = CM_POINT | pid;
        continue;
      }
      const uint32_t id = atomicAdd(&C->nsegs[p ^ 1], 1u);
      if (id >= caps.segs) { set_status(C, GGMS_E_INTERNAL); continue; }
      Seg<K> c;
      c.off = s.off + start;
      c.cnt = cnt;
      c.lo = blo;
      c.hi = bhi;
      c.shift = (uint32_t)max(0, bitlen((K)(bhi - blo)) - RADIX_BITS);
      c.small = cnt <= caps.small_keys ? 1u : 0u;
      c.pad = 0u;
      segs_q[id] = c;
      cursor_q[id] = 0u;
      khead_q[id] = K_NIL;
      out[u] = id;
      if (c.small) {
        const bool tiny = cnt <= caps.tiny_keys;
        const uint32_t si = atomicAdd(tiny ? &C->ntiny : &C->nsmall, 1u);
        if (si < caps.segs) (tiny ? tinies : smalls)[si] = id; else set_status(C, GGMS_E_INTERNAL);
        continue;
      }
      const uint32_t bi = atomicAdd(&C->nbig[p ^ 1], 1u);
      if (bi < caps.segs) bigs_q[bi] = id; else set_status(C, GGMS_E_INTERNAL);
      const uint32_t nt = (cnt + TILE - 1) / TILE;
      const uint32_t t0 = atomicAdd(&C->ntiles[p ^ 1], nt);
      if (t0 + nt > caps.tiles || t0 + nt < t0) { set_status(C, GGMS_E_INTERNAL); continue; }
      for (uint32_t t = 0; t < nt; ++t) tiles_q[t0 + t] = TileRef{id, t};
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < PER; ++u) I[threadIdx.x + u * NT] = out[u];
    __syncthreads();
  }
}

// Copies each key whose bin became a child segment into that child's region.
// Tiles go to CTAs grid-stride, so the CTAs running at one time fill the same
// children side by side and L2 merges their partial sectors (contiguous tile
// ranges per CTA measured 24 % slower on the 4096-segment batch).
template <typename InT, int NT, bool Q = false>
__global__ __launch_bounds__(NT) void lvl_compact(const InT* __restrict__ src,
                                                 const Seg<typename KeyOf<InT>::K>* __restrict__ segs,
                                                 const TileRef* __restrict__ tiles,
                                                 const Counters* __restrict__ C, int p,
                                                 const uint32_t* __restrict__ rows,
                                                 const Seg<typename KeyOf<InT>::K>* __restrict__ segs_q,
                                                 uint32_t* cursor_q, typename KeyOf<InT>::K* dst,
                                                 Caps caps, const typename KeyOf<InT>::K* __restrict__ qtab,
                                                 const uint16_t* __restrict__ qdir) {
  pdl_entry();
  using K = typename KeyOf<InT>::K;
  __shared__ uint32_t cm[NBIN];
  __shared__ __align__(16) K qb[Q ? QB : 1];
  __shared__ __align__(16) uint16_t qd[Q ? QDS : 8];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nt = min(C->ntiles[p], caps.tiles);
  const uint32_t ns = min(C->nsegs[p], caps.segs);
  if (Q && nt && blockIdx.x == 0 && threadIdx.x == 0)  // level 0 reads the input
    atomicAdd(&const_cast<Counters*>(C)->passes, 1u);
  uint32_t loaded = 0xFFFFFFFFu;  // segment whose child map (and table) is in shared memory
  for (uint32_t t = blockIdx.x; t < nt; t += gridDim.x) {
    const TileRef tr = tiles[t];
    if (tr.seg >= ns) continue;  // only after a capacity error (status already set)
    const Seg<K> s = segs[tr.seg];
    if (tr.seg != loaded) {  // the previous tile ended with a barrier
      const uint32_t* row = rows + (size_t)tr.seg * NBIN;
      for (uint32_t i = threadIdx.x; i < NBIN; i += NT) cm[i] = row[i];
      if (Q) qtab_to_smem<K>(qtab, qdir, s.pad, qb, qd);
      loaded = tr.seg;
    }
    __syncthreads();
    const uint64_t beg = s.off + (uint64_t)tr.no * TILE;
    const uint64_t end = min(beg + TILE, s.off + s.cnt);
    constexpr int U = 4;  // loads in flight per thread before the warp-synchronous part
    const uint64_t span = ((end - beg + NT * U - 1) / (NT * U)) * (NT * U);
    for (uint64_t o = threadIdx.x; o < span; o += NT * U) {
      K kk[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint64_t i = beg + o + (uint64_t)u * NT;
        kk[u] = i < end ? KeyOf<InT>::to(src[i]) : (K)0;
      }
      // 1. each key's child (CM_NONE when its bin is not copied)
      uint32_t cc[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        cc[u] = CM_NONE;
        if (beg + o + (uint64_t)u * NT < end) {
          uint32_t bin;
          if (Q) bin = qbin<K>(kk[u], s.lo, s.shift, qb, qd);
          else bin = min((uint32_t)((K)(kk[u] - s.lo) >> s.shift), (uint32_t)NBIN - 1u);
          cc[u] = cm[bin];
        }
      }
      // 2. one cursor reservation per group of lanes with the same child, for
      // all U keys before any result is used: the U global atomics of a warp
      // are in flight together instead of one round trip after another
      uint32_t peers[U], base[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool hit = cc[u] < CM_POINT;
        const uint32_t hm = __ballot_sync(FULL, hit);
        peers[u] = 0u;
        base[u] = 0u;
        if (hit) {
          peers[u] = __match_any_sync(hm, cc[u]);
          if ((int)lane == __ffs(peers[u]) - 1) base[u] = atomicAdd(&cursor_q[cc[u]], (uint32_t)__popc(peers[u]));
        }
      }
      // 3. the stores
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (peers[u]) {
          const uint32_t b0 = __shfl_sync(peers[u], base[u], __ffs(peers[u]) - 1);
          const uint32_t slot = b0 + __popc(peers[u] & lanemask_lt());
          const Seg<K>& sg = segs_q[cc[u]];
          if (slot < sg.cnt) dst[sg.off + slot] = kk[u];
          else set_status(const_cast<Counters*>(C), GGMS_E_INTERNAL);
        }
      }
    }
    __syncthreads();
  }
}



// ------------------------------------------------------------------ small segments
// One CTA finishes a whole small segment in shared memory: its keys (as
// offsets from the segment's lo) are loaded once, then a radix select with
// 8-bit digits runs for up to SS_GROUP ks at a time (one 256-bin histogram per
// k, built from the keys that still match the k's prefix); a segment with more
// than SS_SORT_ABOVE ks is bitonic-sorted in place once instead.  The ks of the
// segment come from the lock-free list the relabel step built.
constexpr int SS_GROUP = 16;
constexpr int SS_MAXK = 256;
constexpr int SS_SORT_ABOVE = 64;   // more ks than this in one segment: bitonic sort instead

template <typename InT, int NT>
__global__ __launch_bounds__(NT) void small_select(const InT* __restrict__ src,
                                                  const Seg<typename KeyOf<InT>::K>* __restrict__ segs_q,
                                                  const uint32_t* __restrict__ smalls,
                                                  const Counters* __restrict__ C_,
                                                  const uint32_t* __restrict__ khead_q,
                                                  const uint32_t* __restrict__ knext,
                                                  const int64_t* __restrict__ k_off,
                                                  const uint32_t* __restrict__ k_rank, uint32_t* k_seg,
                                                  typename KeyOf<InT>::K* k_key, uint32_t small_keys,
                                                  Caps caps) {
  pdl_entry();
  using K = typename KeyOf<InT>::K;
  Counters* C = const_cast<Counters*>(C_);
  extern __shared__ __align__(128) uint8_t smem[];
  K* vals = (K*)smem;
  uint32_t* hist = (uint32_t*)(smem + SMALL_SMEM);           // [SS_GROUP][256]
  __shared__ uint32_t kid[SS_MAXK];
  __shared__ uint32_t nk_s, next_s, kend_s;
  __shared__ uint32_t rk[SS_GROUP];
  __shared__ K pk[SS_GROUP];
  __shared__ K upk[SS_GROUP];       // distinct prefixes of the current round
  __shared__ uint32_t hmap[SS_GROUP];  // k -> its prefix's histogram
  __shared__ uint32_t nuniq;
  GGMS_TRACE(35);
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t ns = min(C->nsmall, caps.segs);
  for (uint32_t t = blockIdx.x; t < ns; t += gridDim.x) {
    const uint32_t id = smalls[t];
    const Seg<K> s = segs_q[id];
    const uint32_t cnt = min(s.cnt, small_keys);
    if (s.cnt > small_keys) set_status(C, GGMS_E_INTERNAL);
    for (uint32_t i0 = tid; i0 < cnt; i0 += 8 * NT) {  // eight independent loads in flight
      K v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const uint32_t i = i0 + q * NT;
        v[q] = i < cnt ? KeyOf<InT>::to(src[s.off + i]) : s.lo;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const uint32_t i = i0 + q * NT;
        if (i < cnt) vals[i] = (K)(v[q] - s.lo);
      }
    }
    const int bits = bitlen((K)(s.hi - s.lo));
    bool sorted_seg = false;
    if (tid == 0) {  // the ks: the segment's list, or (k_off: a caller segment) its k range
      if (k_off) {
        const uint32_t k0 = (uint32_t)k_off[id], k1 = (uint32_t)k_off[id + 1];
        next_s = k0 < k1 ? k0 : K_NIL;
        kend_s = k1;
      } else {
        next_s = khead_q[id];
      }
    }
    __syncthreads();
    while (next_s != K_NIL) {
      __syncthreads();
      if (k_off) {  // the next up to SS_MAXK ks of the range
        const uint32_t k0 = next_s, m = min((uint32_t)SS_MAXK, kend_s - k0);
        for (uint32_t j = tid; j < m; j += NT) kid[j] = k0 + j;
        __syncthreads();
        if (tid == 0) {
          nk_s = m;
          next_s = (k0 + m < kend_s) ? k0 + m : K_NIL;
        }
      } else if (tid == 0) {  // collect up to SS_MAXK ks from the list
        uint32_t k = next_s, m = 0;
        while (k != K_NIL && m < (uint32_t)SS_MAXK) { kid[m++] = k; k = knext[k]; }
        nk_s = m;
        next_s = k;
      }
      __syncthreads();
      const uint32_t m = nk_s;
      if (m > (uint32_t)SS_SORT_ABOVE) {
        // many ks in one segment (e.g. a top-k): sort the segment once instead
        if (!sorted_seg) {
          uint32_t N = 1;
          while (N < cnt) N <<= 1;
          for (uint32_t i = cnt + tid; i < N; i += NT) vals[i] = key_max<K>();
          __syncthreads();
          for (uint32_t kk = 2; kk <= N; kk <<= 1) {
            for (uint32_t jj = kk >> 1; jj > 0; jj >>= 1) {
              for (uint32_t i = tid; i < N; i += NT) {
                const uint32_t ixj = i ^ jj;
                if (ixj > i) {
                  const K a = vals[i], b = vals[ixj];
                  if ((a > b) == ((i & kk) == 0)) { vals[i] = b; vals[ixj] = a; }
                }
              }
              __syncthreads();
            }
          }
          sorted_seg = true;
        }
        for (uint32_t j = tid; j < m; j += NT) {
          const uint32_t k = kid[j];
          const uint32_t r = k_rank[k];
          if (r < cnt) k_key[k] = (K)(s.lo + vals[r]);
          else set_status(C, GGMS_E_INTERNAL);
          k_seg[k] = K_DONE;
        }
        __syncthreads();
        continue;
      }
      for (uint32_t g0 = 0; g0 < m; g0 += SS_GROUP) {
        const uint32_t g = min((uint32_t)SS_GROUP, m - g0);
        if (tid < g) {
          rk[tid] = k_rank[kid[g0 + tid]];
          pk[tid] = 0;
        }
        // digits of 8 bits from the top of the segment's range: v < 2^bits
        for (int top = bits; top > 0;) {
          const int width = min(8, top);
          const int sh = top - width;
          const uint32_t dmask = (1u << width) - 1u;
          __syncthreads();
          if (tid == 0) {  // ks with the same prefix share one histogram
            uint32_t h = 0;
            for (uint32_t j = 0; j < g; ++j) {
              uint32_t u = 0;
              while (u < h && upk[u] != pk[j]) ++u;
              if (u == h) upk[h++] = pk[j];
              hmap[j] = u;
            }
            nuniq = h;
          }
          __syncthreads();
          const uint32_t h = nuniq;
          for (uint32_t i = tid; i < h * 256; i += NT) hist[i] = 0u;
          __syncthreads();
          for (uint32_t i = tid; i < cnt; i += NT) {
            const K v = vals[i];
            for (uint32_t u = 0; u < h; ++u) {
              if ((((v ^ upk[u]) >> sh) >> width) == 0) {  // same bits above this digit
                atomicAdd(&hist[u * 256 + (uint32_t)((v >> sh) & dmask)], 1u);
                break;  // prefixes of one length are disjoint
              }
            }
          }
          __syncthreads();
          if (warp < g) {  // warp j picks the digit holding rank rk[j]
            const uint32_t j = warp;
            const uint32_t* hj = hist + hmap[j] * 256;
            uint32_t c8[8], sum = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) { c8[q] = hj[lane * 8 + q]; sum += c8[q]; }
            uint32_t inc = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const uint32_t tt = __shfl_up_sync(FULL, inc, o);
              if ((int)lane >= o) inc += tt;
            }
            const uint32_t r = rk[j];
            const uint32_t before = inc - sum;
            const bool mine = before <= r && r < inc;
            const uint32_t who = __ballot_sync(FULL, mine);
            if (mine) {
              uint32_t cum = before, d = lane * 8;
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                if (r < cum + c8[q]) { d = lane * 8 + q; break; }
                cum += c8[q];
              }
              rk[j] = r - cum;
              pk[j] = pk[j] | ((K)d << sh);
            }
            if (who == 0 && lane == 0) set_status(C, GGMS_E_INTERNAL);  // rank beyond the segment
          }
          top = sh;
        }
        __syncthreads();
        if (tid < g) {
          const uint32_t k = kid[g0 + tid];
          k_key[k] = (K)(s.lo + pk[tid]);
          k_seg[k] = K_DONE;
        }
        __syncthreads();
      }
    }
    if (tid == 0) atomicAdd(&C->small_segs, 1u);
    __syncthreads();
  }
  GGMS_TRACE(36);
  GGMS_TRACE_CTA(4);
}

// One warp finishes a whole tiny segment (at most tiny_keys<K>() keys, as
// offsets from its lo, in the warp's slice of shared memory).  With few ks: per
// k, a radix select with 8-bit digits from the top of the segment's range (one
// warp-private 256-bin histogram per digit).  With more than TS_SORT_ABOVE ks
// (caller segments of the batched path): the slice is bitonic-sorted once and
// the lanes read their ks' answers from it.  The ks come from the segment's
// list, or (k_off given: the segments are the caller's) from its k range.
constexpr int TS_NT = 128;

template <typename K>
__device__ __forceinline__ K warp_radix_select(const K* v, uint32_t cnt, int bits, uint32_t r, uint32_t* h,
                                               uint32_t lane, bool* ok) {
  K pre = 0;
  for (int top = bits; top > 0;) {
    const int width = min(8, top);
    const int sh = top - width;
    const uint32_t dmask = (1u << width) - 1u;
#pragma unroll
    for (int q = 0; q < 8; ++q) h[lane * 8 + q] = 0u;
    __syncwarp();
    for (uint32_t i = lane; i < cnt; i += 32) {
      const K x = v[i];
      if ((((x ^ pre) >> sh) >> width) == 0) atomicAdd(&h[(uint32_t)(x >> sh) & dmask], 1u);
    }
    __syncwarp();
    uint32_t c8[8], sum = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) { c8[q] = h[lane * 8 + q]; sum += c8[q]; }
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t tt = __shfl_up_sync(FULL, inc, o);
      if ((int)lane >= o) inc += tt;
    }
    const uint32_t before = inc - sum;
    const bool mine = before <= r && r < inc;
    const uint32_t who = __ballot_sync(FULL, mine);
    uint32_t d = 0, nr = 0;
    if (mine) {
      uint32_t cum = before;
      d = lane * 8 + 7;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if (r < cum + c8[q]) { d = lane * 8 + q; break; }
        cum += c8[q];
      }
      nr = r - cum;
    }
    const int owner = who ? __ffs(who) - 1 : 0;
    d = __shfl_sync(FULL, d, owner);
    nr = __shfl_sync(FULL, nr, owner);
    __syncwarp();  // every lane has read the histogram before the next digit clears it
    if (!who) {    // rank beyond the segment (warp-uniform)
      *ok = false;
      return pre;
    }
    r = nr;
    pre = pre | ((K)d << sh);
    top = sh;
  }
  *ok = true;
  return pre;
}

template <typename InT, int NT>
__global__ __launch_bounds__(NT) void tiny_select(const InT* __restrict__ src,
                                                 const Seg<typename KeyOf<InT>::K>* __restrict__ segs_q,
                                                 const uint32_t* __restrict__ tinies,
                                                 const Counters* __restrict__ C_,
                                                 const uint32_t* __restrict__ khead_q,
                                                 const uint32_t* __restrict__ knext,
                                                 const int64_t* __restrict__ k_off,
                                                 const uint32_t* __restrict__ k_rank, uint32_t* k_seg,
                                                 typename KeyOf<InT>::K* k_key, Caps caps) {
  // Launched right after small_select, whose output it does not read: it lets
  // its successor launch and runs beside small_select, and waits for it only
  // at its end (so that it completes after its predecessor).
  pdl_trigger();
  using K = typename KeyOf<InT>::K;
  constexpr uint32_t TK = tiny_keys<K>();
  constexpr int NW = NT / 32;
  __shared__ K buf[NW][TK];
  __shared__ uint32_t hist[NW][256];
  Counters* C = const_cast<Counters*>(C_);
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  K* v = buf[wid];
  uint32_t* h = hist[wid];
  const uint32_t nt = min(C->ntiny, caps.segs);
  // a warp takes up to 32 list entries at a time (fewer when the list is short,
  // so that every warp gets work): lane j loads entry j's descriptor and k-list
  // head -- the chain of dependent loads is paid once per batch -- then the warp
  // finishes the segments one by one
  GGMS_TRACE(39);
  const uint32_t nwarps = gridDim.x * NW;
  const uint32_t batch = max(1u, min(32u, nt / nwarps));
  for (uint32_t t0 = (blockIdx.x * NW + wid) * batch; t0 < nt; t0 += nwarps * batch) {
    const uint32_t tj = t0 + lane;
    uint32_t pid = 0u, pkh = K_NIL;
    Seg<K> ps{};
    if (lane < batch && tj < nt) {
      pid = tinies[tj];
      ps = segs_q[pid];
      if (!k_off) pkh = khead_q[pid];
    }
    const uint32_t nb = min(batch, nt - t0);
    for (uint32_t j = 0; j < nb; ++j) {
      const uint32_t id = __shfl_sync(FULL, pid, j);
      Seg<K> s;
      s.off = __shfl_sync(FULL, ps.off, j);
      s.cnt = __shfl_sync(FULL, ps.cnt, j);
      s.lo = __shfl_sync(FULL, ps.lo, j);
      s.hi = __shfl_sync(FULL, ps.hi, j);
      const uint32_t khead = __shfl_sync(FULL, pkh, j);
      const uint32_t cnt = s.cnt;
      if (cnt > TK) {  // cannot happen: tiny segments are created with cnt <= tiny_keys
        if (lane == 0) set_status(C, GGMS_E_INTERNAL);
        continue;
      }
      for (uint32_t i0 = lane; i0 < cnt; i0 += 32 * 8) {  // eight independent loads in flight
        K x[8];
  #pragma unroll
        for (int q = 0; q < 8; ++q) {
          const uint32_t i = i0 + q * 32;
          x[q] = i < cnt ? KeyOf<InT>::to(src[s.off + i]) : s.lo;
        }
  #pragma unroll
        for (int q = 0; q < 8; ++q) {
          const uint32_t i = i0 + q * 32;
          if (i < cnt) v[i] = (K)(x[q] - s.lo);
        }
      }
      __syncwarp();
      const int bits = bitlen((K)(s.hi - s.lo));
      // Up to 64 keys: every key's rank by comparing it with all the others (ties
      // broken by position), once for all of the segment's ks; a k is then one
      // ballot.  Cheaper than 8-bit radix rounds, whose 256-bin histograms cost
      // the same however few keys there are.
      const bool by_rank = cnt <= 64u;
      uint32_t ra = 0xFFFFFFFFu, rb = 0xFFFFFFFFu;
      K ka = 0, kb = 0;
      if (by_rank) {
        ka = lane < cnt ? v[lane] : (K)0;
        kb = lane + 32u < cnt ? v[lane + 32u] : (K)0;
        uint32_t ca = 0, cb = 0;
        for (uint32_t j = 0; j < cnt; ++j) {
          const K x = v[j];
          ca += (x < ka || (x == ka && j < lane)) ? 1u : 0u;
          cb += (x < kb || (x == kb && j < lane + 32u)) ? 1u : 0u;
        }
        if (lane < cnt) ra = ca;
        if (lane + 32u < cnt) rb = cb;
      }
      auto rank_pick = [&](uint32_t r, bool* ok) -> K {
        const uint32_t ma = __ballot_sync(FULL, ra == r), mb = __ballot_sync(FULL, rb == r);
        *ok = (ma | mb) != 0u;
        const K xa = __shfl_sync(FULL, ka, ma ? __ffs(ma) - 1 : 0);
        const K xb = __shfl_sync(FULL, kb, mb ? __ffs(mb) - 1 : 0);
        return ma ? xa : xb;
      };
      if (k_off && by_rank) {
        const int64_t k0 = k_off[id], k1 = k_off[id + 1];
        for (int64_t k = k0; k < k1; ++k) {
          if (k_seg[k] == K_DONE) continue;  // warp-uniform
          bool ok = false;
          const K pre = rank_pick(k_rank[k], &ok);
          if (lane == 0) {
            if (ok) k_key[k] = (K)(s.lo + pre); else set_status(C, GGMS_E_INTERNAL);
            k_seg[k] = K_DONE;
          }
        }
      } else if (k_off) {
        const int64_t k0 = k_off[id], k1 = k_off[id + 1];
        if ((uint64_t)(k1 - k0) > TS_SORT_ABOVE) {
          uint32_t N = 32;
          while (N < cnt) N <<= 1;
          for (uint32_t i = cnt + lane; i < N; i += 32) v[i] = key_max<K>();
          __syncwarp();
          for (uint32_t kk = 2; kk <= N; kk <<= 1) {
            for (uint32_t jj = kk >> 1; jj > 0; jj >>= 1) {
              for (uint32_t i = lane; i < N; i += 32) {
                const uint32_t ixj = i ^ jj;
                if (ixj > i) {
                  const K a = v[i], b = v[ixj];
                  if ((a > b) == ((i & kk) == 0)) { v[i] = b; v[ixj] = a; }
                }
              }
              __syncwarp();
            }
          }
          for (int64_t k = k0 + lane; k < k1; k += 32) {
            if (k_seg[k] == K_DONE) continue;  // an invalid k (status already set)
            const uint32_t r = k_rank[k];
            if (r < cnt) k_key[k] = (K)(s.lo + v[r]); else set_status(C, GGMS_E_INTERNAL);
            k_seg[k] = K_DONE;
          }
        } else {
          for (int64_t k = k0; k < k1; ++k) {
            if (k_seg[k] == K_DONE) continue;  // warp-uniform
            bool ok = false;
            const uint32_t r = k_rank[k];
            const K pre = r < cnt ? warp_radix_select<K>(v, cnt, bits, r, h, lane, &ok) : (K)0;
            if (lane == 0) {
              if (ok) k_key[k] = (K)(s.lo + pre); else set_status(C, GGMS_E_INTERNAL);
              k_seg[k] = K_DONE;
            }
          }
        }
      } else {
        for (uint32_t k = khead; k != K_NIL; k = knext[k]) {
          bool ok = false;
          const uint32_t r = k_rank[k];
          const K pre = by_rank ? rank_pick(r, &ok)
                                : (r < cnt ? warp_radix_select<K>(v, cnt, bits, r, h, lane, &ok) : (K)0);
          if (lane == 0) {
            if (ok) k_key[k] = (K)(s.lo + pre); else set_status(C, GGMS_E_INTERNAL);
            k_seg[k] = K_DONE;
          }
        }
      }
      __syncwarp();  // the slice is reloaded by the warp's next segment
    }
    if (lane == 0) atomicAdd(&C->small_segs, nb);
  }
  GGMS_TRACE(40);
  GGMS_TRACE_CTA(5);
  pdl_wait();
}

// ------------------------------------------------------------------ batched segments
// Level 0 of the batched mode.  A caller segment that holds a k is finished
// directly from the input when it is small (tiny_select for tiny ones,
// small_select below QSAMP keys); a larger one gets quantile bins (seg_sample
// fills its table) and tiles for the level-0 count -- its children then hold
// about 1/QB of it, mostly a single k each.
template <typename K>
__global__ void seg_init(const int64_t* __restrict__ seg_off, uint32_t nseg,
                         const int64_t* __restrict__ k_off, Seg<K>* segs0, TileRef* tiles0,
                         uint32_t* khead0, uint32_t* smalls, uint32_t* tinies, uint32_t* bigs0,
                         uint32_t cap_q, Counters* C, Caps caps) {
  pdl_entry();
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const int64_t a = seg_off[s], b = seg_off[s + 1];
  Seg<K> d;
  d.off = (uint64_t)a;
  d.cnt = (b > a) ? (uint32_t)(b - a) : 0u;
  d.lo = 0;
  d.hi = key_max<K>();
  d.shift = 0u;
  d.small = 0u;
  d.pad = 0u;
  khead0[s] = K_NIL;
  if (b < a) set_status(C, GGMS_E_INVALID_ARG);
  if (k_off[s + 1] == k_off[s] || d.cnt == 0) {  // nothing to select here
    d.small = 1u;  // no row, no tiles
    segs0[s] = d;
    return;
  }
  if (d.cnt <= caps.tiny_keys || d.cnt < QSAMP) {
    d.small = 1u;
    segs0[s] = d;
    const bool tiny = d.cnt <= caps.tiny_keys;
    const uint32_t si = atomicAdd(tiny ? &C->ntiny : &C->nsmall, 1u);
    if (si < caps.segs) (tiny ? tinies : smalls)[si] = s; else set_status(C, GGMS_E_INTERNAL);
    return;
  }
  const uint32_t q = atomicAdd(&C->nbig[0], 1u);  // its quantile table: q
  if (q < caps.segs) bigs0[q] = s;
  if (q >= cap_q) {  // cannot happen: cap_q bounds the segments of QSAMP keys or more
    set_status(C, GGMS_E_INTERNAL);
    d.small = 1u;
    segs0[s] = d;
    return;
  }
  d.pad = q;
  segs0[s] = d;
  const uint32_t nt = (d.cnt + TILE - 1) / TILE;
  const uint32_t t0 = atomicAdd(&C->ntiles[0], nt);
  if (t0 + nt > caps.tiles) { set_status(C, GGMS_E_INTERNAL); return; }
  for (uint32_t t = 0; t < nt; ++t) tiles0[t0 + t] = TileRef{s, t};
}

__global__ void seg_set_count(Counters* C, uint32_t nseg) {
  pdl_entry(); C->nsegs[0] = nseg; }

// k i belongs to the segment s with k_off[s] <= i < k_off[s+1]; the ks of a
// segment that is finished directly go on its list.
template <typename K>
__global__ void k_init_seg(const uint32_t* __restrict__ ks, uint32_t nk,
                           const int64_t* __restrict__ seg_off, const int64_t* __restrict__ k_off,
                           uint32_t nseg, const Seg<K>* __restrict__ segs0, uint32_t* khead0,
                           uint32_t* knext, uint32_t* k_rank, uint32_t* k_seg, Counters* C) {
  pdl_entry();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nk) return;
  uint32_t lo = 0, hi = nseg - 1;  // largest s with k_off[s] <= i
  while (lo < hi) {
    uint32_t m = (lo + hi + 1) >> 1;
    if (k_off[m] <= (int64_t)i) lo = m; else hi = m - 1;
  }
  const uint64_t len = (uint64_t)(seg_off[lo + 1] - seg_off[lo]);
  const uint32_t k = ks[i];
  if (k < 1u || (uint64_t)k > len) {
    set_status(C, GGMS_E_INVALID_ARG);
    k_seg[i] = K_DONE;
    k_rank[i] = 0;
    return;
  }
  k_rank[i] = (uint32_t)(len - k);
  k_seg[i] = lo;
  if (segs0[lo].small) knext[i] = atomicExch(&khead0[lo], i);  // lock-free push
}

// ------------------------------------------------------------------ outputs
template <typename T>
__global__ void write_out(const typename KeyOf<T>::K* __restrict__ k_key,
                          const uint32_t* __restrict__ k_seg, uint32_t nk, T* out, Counters* C) {
  pdl_entry();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  GGMS_TRACE(37);
  if (i >= nk) return;
  if (k_seg[i] != K_DONE) set_status(C, GGMS_E_NOT_CONVERGED);
  out[i] = KeyOf<T>::from(k_key[i]);
}

GGMS_END
