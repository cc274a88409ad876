// ggms_internal.cuh -- shared device definitions of the selector.
//
// Keys.  Every input type is mapped on load to an unsigned key whose integer
// order is the value order (the reference compares raw values with >= against
// pivots, DistributedSMOS/bucketMultiselect.cu:178-185; mapping to keys makes
// NaN, -0.0/+0.0 and duplicates exact and lets every later step be integer
// work):
//   float  : bits ^ (negative ? 0xFFFFFFFF : 0x80000000)
//   double : the 64-bit analogue
//   int32  : bits ^ 0x80000000
//   uint32 : identity
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

// Kernels and the host code that launches them are compiled once per value
// type, each translation unit in its own inline namespace ggms::GGMS_TU, so
// no two units share a kernel (or the flag that records that its launch
// attributes were set).  The types and inline helpers below are shared.
#ifndef GGMS_TU
#define GGMS_TU tu_default
#endif
#define GGMS_BEGIN namespace ggms { inline namespace GGMS_TU {
#define GGMS_END } }

// Set-up tracing for development builds only (-DGGMS_SETUP_TRACE): thread 0
// of block 0 stores %globaltimer at numbered points of the kernels into this
// unit's ggms_trace_buf (ggms_f32.cu exports a reader in such builds).
// Compiled out otherwise.
#ifdef GGMS_SETUP_TRACE
static __device__ unsigned long long ggms_trace_buf[64];
#define GGMS_TRACE(i)                                                  \
  do {                                                                 \
    if (threadIdx.x == 0 && blockIdx.x == 0) {                         \
      unsigned long long t_;                                           \
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_));           \
      ggms_trace_buf[(i)] = t_;                                        \
    }                                                                  \
  } while (0)
// Per-CTA points of the two passes: thread 0 of every block stores its
// %globaltimer in row i (0/1 PASS 1 start/end, 2/3 PASS 2 start/end, 4/5 end of
// the CTA and warp finishers).
static __device__ unsigned long long ggms_trace_cta[6][1024];
#define GGMS_TRACE_CTA(i)                                              \
  do {                                                                 \
    if (threadIdx.x == 0 && blockIdx.x < 1024) {                       \
      unsigned long long t_;                                           \
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_));           \
      ggms_trace_cta[(i)][blockIdx.x] = t_;                            \
    }                                                                  \
  } while (0)
#else
#define GGMS_TRACE(i) \
  do {                \
  } while (0)
#define GGMS_TRACE_CTA(i) \
  do {                    \
  } while (0)
#endif

namespace ggms {

// ------------------------------------------------------------------ programmatic dependent launch
// The host launches the kernels of one call with programmatic stream
// serialization, so that a kernel can be scheduled while the one before it on
// the stream is still finishing.  Every kernel therefore begins here: it waits
// for the grids it depends on to complete (their memory visible) before it
// reads or writes anything, then lets the next kernel begin launching.  For a
// kernel launched without that attribute both instructions are no-ops.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// The two halves, for kernels that read data older than their predecessor's
// output before waiting: a kernel's CTAs start only after its predecessor has
// passed its own wait, i.e. after the kernel before that has completed, so
// anything written two or more kernels back may be read before pdl_wait().
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ------------------------------------------------------------------ key traits
template <typename T> struct KeyOf;
template <> struct KeyOf<float> {
  using K = uint32_t;
  static constexpr int BITS = 32;
  __host__ __device__ static K to(float v) {
#ifdef __CUDA_ARCH__
    uint32_t u = __float_as_uint(v);
#else
    uint32_t u; __builtin_memcpy(&u, &v, 4);
#endif
    return u ^ ((u >> 31) ? 0xFFFFFFFFu : 0x80000000u);
  }
  __host__ __device__ static float from(K k) {
    uint32_t u = k ^ ((k >> 31) ? 0x80000000u : 0xFFFFFFFFu);
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float v; __builtin_memcpy(&v, &u, 4); return v;
#endif
  }
};
template <> struct KeyOf<double> {
  using K = uint64_t;
  static constexpr int BITS = 64;
  __host__ __device__ static K to(double v) {
#ifdef __CUDA_ARCH__
    uint64_t u = (uint64_t)__double_as_longlong(v);
#else
    uint64_t u; __builtin_memcpy(&u, &v, 8);
#endif
    return u ^ ((u >> 63) ? 0xFFFFFFFFFFFFFFFFull : 0x8000000000000000ull);
  }
  __host__ __device__ static double from(K k) {
    uint64_t u = k ^ ((k >> 63) ? 0x8000000000000000ull : 0xFFFFFFFFFFFFFFFFull);
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double v; __builtin_memcpy(&v, &u, 8); return v;
#endif
  }
};
template <> struct KeyOf<uint32_t> {
  using K = uint32_t;
  static constexpr int BITS = 32;
  __host__ __device__ static K to(uint32_t v) { return v; }
  __host__ __device__ static uint32_t from(K k) { return k; }
};
template <> struct KeyOf<uint64_t> {  // keys of 64-bit types are already keys
  using K = uint64_t;
  static constexpr int BITS = 64;
  __host__ __device__ static K to(uint64_t v) { return v; }
  __host__ __device__ static uint64_t from(K k) { return k; }
};
template <> struct KeyOf<int32_t> {
  using K = uint32_t;
  static constexpr int BITS = 32;
  __host__ __device__ static K to(int32_t v) { return ((uint32_t)v) ^ 0x80000000u; }
  __host__ __device__ static int32_t from(K k) { return (int32_t)(k ^ 0x80000000u); }
};

template <typename K> struct KeyBits;
template <> struct KeyBits<uint32_t> { static constexpr int value = 32; };
template <> struct KeyBits<uint64_t> { static constexpr int value = 64; };

__device__ __forceinline__ float key_to_float_rn(uint32_t d) { return __uint2float_rn(d); }
__device__ __forceinline__ float key_to_float_rn(uint64_t d) { return __ull2float_rn(d); }

__host__ __device__ __forceinline__ int bitlen(uint32_t v) {
#ifdef __CUDA_ARCH__
  return 32 - __clz(v);
#else
  return v ? 32 - __builtin_clz(v) : 0;
#endif
}
__host__ __device__ __forceinline__ int bitlen(uint64_t v) {
#ifdef __CUDA_ARCH__
  return 64 - __clzll((long long)v);
#else
  return v ? 64 - __builtin_clzll(v) : 0;
#endif
}

// ------------------------------------------------------------------ constants
constexpr int RADIX_BITS = 11;                  // bits resolved per refinement level
constexpr int NBIN = 1 << RADIX_BITS;           // 2048 bins per refinement segment
constexpr int NBIN_WORDS = NBIN / 32;           // active-flag words per segment row
constexpr int TILE = 16384;                     // elements per refinement work item
constexpr int ASG_MAXM = 1024;                  // max segments of a PL model
constexpr int ASG_CELL_BITS = 12;
constexpr int ASG_NCELL = 1 << ASG_CELL_BITS;   // uniform lookup cells over the knot range
constexpr uint32_t K_DONE = 0xFFFFFFFFu;        // k_seg value of a resolved k
constexpr uint32_t CM_NONE = 0xFFFFFFFFu;       // child-map entry: bin holds no requested k
constexpr uint32_t CM_POINT = 0x80000000u;      // child-map flag: bin is one key; low bits index points[]

// ------------------------------------------------------------------ assigner
// A monotone piecewise-linear map key -> bucket in [0, B).  Keys below the
// first knot go to bucket 0, keys above the last knot to bucket B-1; inside,
// segment j ([x[j], x[j+1])) maps linearly onto buckets [base[j], base[j+1]-1].
// This one format carries both the reference's sampled pivots + slopes
// (DistributedSMOS/bucketMultiselect.cu:421-515, 135-210) and the learned
// CDF models, which are compiled into it.  A uniform cell table over the knot
// range gives the segment of a key in O(1) (plus a short forward walk).
template <typename K>
struct Assigner {
  uint32_t M;                 // segments; knots are x[0..M]
  uint32_t B;                 // buckets
  uint32_t csh;               // cell = (key - x[0]) >> csh
  uint32_t ncell;             // cells in use
  uint32_t kind;              // GGMS_ASSIGNER_* that built it
  float quality;              // imbalance measured on the sample (max/mean)
  float loss;                 // training loss (learned) or 0
  uint32_t pad;
  K x[ASG_MAXM + 1];
  uint32_t base[ASG_MAXM + 1];
  float slope[ASG_MAXM];
  uint16_t idx[ASG_NCELL];
};

// Shared-memory view of an assigner (the hot loops copy it in once).
template <typename K>
struct AsgView {
  const K* x;
  const uint32_t* base;
  const float* slope;
  const uint16_t* idx;
  uint32_t M, B, csh;
};

// The single evaluation routine used by the counting pass, the compaction pass
// and the inverse (bucket -> key range) search.  All arithmetic is explicitly
// rounded (no contraction), so every kernel computes the same bucket.
template <typename K>
__device__ __forceinline__ uint32_t asg_eval(const AsgView<K>& a, K key) {
  const K x0 = a.x[0];
  if (key < x0) return 0u;
  const uint32_t M = a.M;
  if (key > a.x[M]) return a.B - 1u;
  if (M == 0u) return a.base[0];
  uint32_t c = (uint32_t)((key - x0) >> a.csh);
  uint32_t j = a.idx[c];
  while (j + 1u < M && key >= a.x[j + 1u]) ++j;
  const uint32_t b0 = a.base[j];
  // segment j maps into [base[j], base[j+1] - 1]: distinct knots never share a bucket
  const uint32_t span = a.base[j + 1u] - b0;
  const float cap = __uint2float_rn(span ? span - 1u : 0u);
  float t = __fmul_rn(key_to_float_rn((K)(key - a.x[j])), a.slope[j]);
  t = fminf(t, cap);
  return b0 + __float2uint_rz(t);
}


// ------------------------------------------------------------------ compiled grid assigner
// What the two passes evaluate.  Any monotone key -> bucket model (the sampled
// pivots or a learned CDF, both held as a piecewise-linear Assigner above) is
// resampled onto a uniform grid of up to 2^11 cells over the sample's key range,
// with one extra cell below and above for the open tails (buckets 0 and B-1:
// no min/max pass is needed, unlike the reference's thrust::minmax_element,
// DistributedSMOS/bucketMultiselect.cu:543-547).  Keys are clamped into the
// grid, so a key costs: two min/max, one shared-memory lookup (two in one of the
// up-to-32 heaviest cells, which are split into 2^6 sub-cells), and an integer
// interpolation b_c + (offset * (b_{c+1} - b_c)) >> shift -- exact, monotone by
// construction, no search and no floating point.
constexpr int GRID_BITS1 = 11;
constexpr int GRID_NC1 = 1 << GRID_BITS1;       // interior level-1 cells
constexpr int GRID_T1 = GRID_NC1 + 2;           // + the two tail cells
constexpr int GRID_SUBCAP = 2048;               // sub-cell entries shared by all split cells
constexpr int GRID_MAXSB = 10;                  // a split cell has 2^1 .. 2^10 sub-cells
constexpr uint32_t GRID_SPLIT = 0x80000000u;    // entry flag

// entry: .x = bucket at the cell's first key, .y = bucket at the next cell's
// first key; or, for a split cell, .x = GRID_SPLIT | (sub_bits << 16),
// .y = index of its first sub-cell entry (sub-cells are plain entries).
template <typename K>
struct Grid {
  K origin;                    // first key of cell 0
  K gmax;                      // last key of the last cell (keys are clamped to [origin, gmax])
  uint32_t sh1, nsubent, B, ncell, nsplit, kind;
  float quality;               // max/mean occupancy on the sample (256 bucket groups)
  float loss;
  uint32_t pad[2];
  uint2 t1[GRID_T1];
  uint2 t2[GRID_SUBCAP];
};

template <typename K>
struct GridView {
  const uint2* t1;
  const uint2* t2;
  K origin, gmax;
  uint32_t sh1, B;
};

// floor(off * span / 2^sh) for off < 2^sh, span < 2^16: monotone in off, < span.
__device__ __forceinline__ uint32_t grid_lin(uint32_t off, uint32_t span, uint32_t sh) {
  return (uint32_t)(((uint64_t)off * span) >> sh);
}
__device__ __forceinline__ uint32_t grid_lin(uint64_t off, uint32_t span, uint32_t sh) {
  const uint32_t s = min(sh, 32u);  // keep the top 32 bits of the offset
  return (uint32_t)((((uint64_t)(uint32_t)(off >> (sh - s))) * span) >> s);
}

template <typename K>
__device__ __forceinline__ uint32_t grid_eval(const GridView<K>& g, K key) {
  const K kc = min(max(key, g.origin), g.gmax);
  const K d = (K)(kc - g.origin);
  uint2 e = g.t1[(uint32_t)(d >> g.sh1)];
  uint32_t sh = g.sh1;
  if (e.x & GRID_SPLIT) {
    const uint32_t sb = (e.x >> 16) & 31u;
    sh = g.sh1 - sb;
    e = g.t2[e.y + ((uint32_t)(d >> sh) & ((1u << sb) - 1u))];
  }
  if constexpr (sizeof(K) == 4) {
    // floor(off * span / 2^sh) with off = d mod 2^sh: shifting d left by 32 - sh
    // drops the bits above the offset and scales it by 2^(32 - sh), so the high
    // word of the product with span is the same floor.  The clamped funnel
    // shift gives 0 for sh = 0 (a one-key cell, offset 0).
    return e.x + __umulhi(__funnelshift_lc(0u, (uint32_t)d, 32u - sh), e.y - e.x);
  } else {
    const K off = d & (K)(((K)1 << sh) - 1);
    return e.x + grid_lin(off, e.y - e.x, sh);
  }
}

// Smallest key whose grid bucket is >= target (the largest key when no key's is): the
// inverse of the monotone grid function, for the key range of a bucket.  A
// binary search over the cells' first buckets (and over the sub-cells of a
// split cell) finds the cell that holds the answer, and the cell's integer
// interpolation is inverted in closed form: the smallest offset with
// floor(off' * span / 2^s) >= t is off' = ceil(t * 2^s / span).  The result is
// checked with grid_eval at the key and the key before it; should the check
// fail, a binary search over all keys answers, so the result is exact either way.
template <typename K>
__device__ K grid_inv(const GridView<K>& g, uint32_t ncell, uint32_t target) {
  if (grid_eval<K>(g, (K)0) >= target) return (K)0;
  if (grid_eval<K>(g, g.gmax) < target) return (K)~(K)0;
  auto cstart = [&](uint32_t c) -> uint32_t {  // bucket of the cell's first key
    const uint2 e = g.t1[c];
    return (e.x & GRID_SPLIT) ? g.t2[e.y].x : e.x;
  };
  uint32_t lo = 0, hi = ncell - 1u;  // the last cell whose first bucket is below target
  while (lo < hi) {
    const uint32_t m = (lo + hi + 1u) >> 1;
    if (cstart(m) < target) lo = m; else hi = m - 1u;
  }
  uint2 e = g.t1[lo];
  uint32_t sh = g.sh1;
  K first = (K)(g.origin + ((K)lo << g.sh1));
  if (e.x & GRID_SPLIT) {
    const uint32_t sb = (e.x >> 16) & 31u;
    sh = g.sh1 - sb;
    uint32_t l2 = 0, h2 = (1u << sb) - 1u;
    while (l2 < h2) {
      const uint32_t m = (l2 + h2 + 1u) >> 1;
      if (g.t2[e.y + m].x < target) l2 = m; else h2 = m - 1u;
    }
    first = (K)(first + ((K)l2 << sh));
    e = g.t2[e.y + l2];
  }
  const uint32_t span = e.y - e.x, t = target - e.x;  // t >= 1: the cell starts below target
  K cand;
  if (t >= span) {  // every key of the cell is below target: the next cell's first key
    cand = (K)(first + ((K)1 << sh));
  } else {
    const uint32_t s = min(sh, 32u);  // grid_lin interpolates on the top 32 bits of the offset
    // ceil(t * 2^s / span): the quotient (< 2^48) from a double division, then
    // corrected to the exact integer ceiling with two multiplications
    const uint64_t num = (uint64_t)t << s;
    uint64_t top = (uint64_t)ceil(__ddiv_rn((double)num, (double)span));
    if (top * span < num) ++top;
    else if (top > 0u && (top - 1u) * span >= num) --top;
    cand = (K)(first + ((K)top << (sh - s)));
  }
  if (cand != (K)0 && grid_eval<K>(g, cand) >= target && grid_eval<K>(g, (K)(cand - 1u)) < target) return cand;
#ifdef GGMS_SETUP_TRACE
  atomicAdd(&ggms_trace_buf[63], 1ull);  // fallbacks, read by the trace reader
#endif
  K a = 0, b = (K)~(K)0;
  while (a < b) {
    const K mid = a + ((b - a) >> 1);
    if (grid_eval<K>(g, mid) >= target) b = mid; else a = mid + 1u;
  }
  return a;
}

// Largest key whose bucket is <= e (the last key of the bucket range ending at
// e).  When no key reaches bucket e + 1 -- e is the last bucket, or the model
// maps even the largest key below e + 1, as a learned model whose buckets are
// focused on the ks can -- that is the largest key itself; grid_inv's answer
// (the largest key as "none") minus one would drop it from the range.
template <typename K>
__device__ K grid_last_key(const GridView<K>& g, uint32_t ncell, uint32_t e) {
  const K kmax = (K)~(K)0;
  if (e >= g.B - 1u || min(grid_eval<K>(g, kmax), g.B - 1u) <= e) return kmax;
  const K first_above = grid_inv<K>(g, ncell, e + 1u);
  return first_above ? (K)(first_above - 1u) : (K)0;  // 0: even key 0 lies above e (an empty range)
}

// ------------------------------------------------------------------ refinement levels
// A segment of candidates.  Every key of the segment lies in [lo, hi]; its bin
// is (key - lo) >> shift, shift chosen so that bins < NBIN.
template <typename K>
struct Seg {
  uint64_t off;   // first element in the level's source buffer (or input)
  uint32_t cnt;   // elements
  uint32_t shift;
  K lo;
  K hi;
  uint32_t small; // finished by small_select (in shared memory), not by another level
  uint32_t pad;
};

constexpr uint32_t K_NIL = 0xFFFFFFFFu;        // end of a per-segment k list
constexpr size_t SMALL_SMEM = 64 * 1024;         // keys of one small segment in shared memory (a power of two)

struct TileRef {
  uint32_t seg;   // segment id in the level's list
  uint32_t no;    // tile number inside the segment
};

// Device counters (one small block of memory, zeroed per call).
struct Counters {
  uint32_t nsegs[2];          // segments of the level stored in pool p
  uint32_t ntiles[2];
  uint32_t npoints;
  uint32_t status;            // nonzero: internal error code
  uint32_t active0;           // active level-0 buckets
  uint32_t point0;            // of which single-key
  uint32_t levels_run;        // refinement levels that had work
  uint32_t max_bucket0;       // largest level-0 bucket
  uint32_t small_segs;        // segments finished in shared memory (all levels)
  uint32_t nsmall;            // small segments created by the current level
  unsigned long long cand0;   // elements copied by the level-0 compaction
  unsigned long long refine_elems;
  uint32_t asg_choice;        // index of the assigner in use (0 sampled, 1 learned)
  uint32_t win_runs;          // PASS 1 window runs in use (0: no windows)
  uint32_t done;              // a refinement level found no segment: later levels are skipped
  uint32_t ntiny;             // tiny segments created by the current level (batched path)
  uint32_t nbig[2];           // segments of pool p that a level refines (listed in bigs[p])
  uint32_t coarse;            // level 0 copies NGRP groups of buckets (most buckets hold a k)
  uint32_t passes;            // launches that read the whole input (counted by the kernels themselves)
};

// PASS 1 windows (l0_window).  From the sample, every requested k gets a
// range of level-0 buckets that holds it with overwhelming probability; the
// union of those ranges, merged into at most L0_WIN runs, is where PASS 1
// computes buckets.  A key outside every run is only counted, per gap between
// runs, and the gap's count is kept in its first bucket ("gap bucket").  The
// answers never depend on the prediction: a k that lands in a gap finds the
// gap bucket, whose segment is then the whole gap.
constexpr uint32_t L0_WIN = 4;
template <typename K>
struct Windows {
  uint32_t on;                                 // 1: PASS 1 buckets only the runs
  uint32_t R;                                  // runs, 1..L0_WIN
  uint32_t cnt;                                // 1: two or more gaps hold keys (PASS 1 counts per run)
  uint32_t tight;                              // 1: the runs hold at most 1/64 of the sample
  uint32_t rb0[L0_WIN], rb1[L0_WIN];           // bucket range of run r (ascending, disjoint)
  uint32_t gb0[L0_WIN + 1], gb1[L0_WIN + 1];   // bucket range of gap g (gb0 > gb1: empty)
  K lo[L0_WIN], hi[L0_WIN];                    // key range of run r (exactly its buckets' keys)
};

// Bucket of grid bucket b under windows: b inside a run, else its gap bucket.
// Monotone non-decreasing in b.
template <typename K>
__device__ __forceinline__ uint32_t win_map(const Windows<K>& w, uint32_t b) {
  for (uint32_t r = 0; r < w.R; ++r)
    if (b <= w.rb1[r]) return b >= w.rb0[r] ? b : w.gb0[r];
  return w.gb0[w.R];
}

// Last bucket of the level-0 segment that starts at bucket b: the gap's last
// bucket for a gap bucket, b itself otherwise.
template <typename K>
__device__ __forceinline__ uint32_t win_end(const Windows<K>& w, uint32_t b) {
  if (w.on)
    for (uint32_t g = 0; g <= w.R; ++g)
      if (b == w.gb0[g] && w.gb0[g] <= w.gb1[g]) return w.gb1[g];
  return b;
}

// Capacities of the device-side lists; every append checks them and records
// GGMS_E_INTERNAL instead of writing out of bounds.
struct Caps {
  uint32_t segs;
  uint32_t tiles;
  uint32_t points;
  uint32_t small_keys;        // a child with at most this many keys is finished by small_select
  uint32_t tiny_keys;         // ... and with at most this many by tiny_select (one warp); 0: never
};

// Level 0 of the batched path: a caller segment too large for small_select
// gets QB bins whose boundaries are every second key of a sorted sample of
// QSAMP of its keys (equal-mass bins whatever the distribution), and a
// directory of QD cells, uniform in key over the sample's range, that gives
// for each cell the boundaries below its first key -- a key's bin is then a
// short search between two directory entries.
constexpr uint32_t QB = NBIN;                   // bins (QB - 1 boundaries)
constexpr uint32_t QSAMP = 2 * QB;              // sampled keys per segment
constexpr int QD_BITS = 12;
constexpr uint32_t QD = 1u << QD_BITS;          // directory cells
constexpr uint32_t QDS = QD + 8;                // directory stride (QD + 1 entries, 16-byte rows)

// Coarse level 0 (single vector, most buckets hold a k): NGRP groups of
// 2^coarse_shift(B) consecutive buckets (B a power of two >= 2 * NGRP).
constexpr uint32_t NGRP = 256;
__host__ __device__ __forceinline__ uint32_t coarse_shift(uint32_t B) {
  uint32_t l = 0;
  while ((2u << l) <= B) ++l;  // log2(B)
  return l > 8u ? l - 8u : 0u;
}

// Keys of one tiny segment (a warp's shared-memory slice of 8 KB).
template <typename K>
__host__ __device__ constexpr uint32_t tiny_keys() { return 8192u / (uint32_t)sizeof(K); }

}  // namespace ggms
