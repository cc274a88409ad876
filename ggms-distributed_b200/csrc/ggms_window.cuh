// ggms_window.cuh -- PASS 1 windows: where the requested ks can lie.
//
// The reference counts every element into its bucket before it knows which
// buckets matter (DistributedSMOS/bucketMultiselect.cu:135-210, 664-679).
// Here the sorted sample already says roughly where each k lies: if the k-th
// key has ascending rank r, the number of sample keys below it is binomial
// (S, q = (r + 1/2) / n), so the key lies between the sample keys at positions
// S q -+ m, m = z sqrt(S q (1 - q)) + z + 2, except with a probability below
// 10^-9 for the default z = 6 (a miss costs time, never exactness).  Every k thus gets a range of level-0 buckets; their
// union, merged across gaps that hold under 1/256 of the sample into at most
// L0_WIN runs holding at most a quarter of it, is the only place PASS 1 computes
// buckets.  Keys elsewhere are counted per gap between runs (a few compares),
// so when the ks are clustered most of the input skips the bucket
// computation entirely.  Nothing here decides an answer: a k outside every
// run lands in a gap bucket, whose segment is then the whole gap.
#pragma once
#include "ggms_setup.cuh"

GGMS_BEGIN

constexpr uint32_t WIN_MAXRAW = 64;    // runs before merging; more: no windows
constexpr uint32_t WIN_NT = 1024;

constexpr uint32_t WIN_IDX = 64;  // every WIN_IDX-th sample key is kept in shared memory

template <typename K>
__host__ __device__ constexpr size_t l0_window_smem(uint32_t B) {
  return GRID_SMEM + sizeof(K) * (65536u / WIN_IDX) + 4u * ((size_t)B / 32u) + 4u * ((size_t)B + 1u);
}

// One CTA.  Dynamic shared memory: l0_window_smem<K>(B) -- the grid (every
// search below evaluates it many times), a coarse index of the sample, a
// bitmap of the B buckets and a difference array over them.
template <typename K>
__global__ __launch_bounds__(WIN_NT) void l0_window(const K* __restrict__ sorted, uint32_t S,
                                                   const uint32_t* __restrict__ krank, uint32_t nk,
                                                   uint64_t n, const Grid<K>* __restrict__ Gs,
                                                   Counters* C, float z, Windows<K>* W) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem[];
  uint2* s1 = reinterpret_cast<uint2*>(smem);
  uint2* s2 = s1 + GRID_T1;
  K* sidx = reinterpret_cast<K*>(smem + GRID_SMEM);                         // sorted[j * WIN_IDX]
  uint32_t* bm = reinterpret_cast<uint32_t*>(sidx + 65536u / WIN_IDX);      // buckets some k may hold
  __shared__ uint32_t red[33];
  __shared__ uint32_t rs[WIN_MAXRAW], re[WIN_MAXRAW], ss[WIN_MAXRAW], se[WIN_MAXRAW];
  __shared__ Windows<K> sw;
  const uint32_t tid = threadIdx.x;
  GGMS_TRACE(17);
  const GridView<K> gv = grid_to_smem<K>(Gs + C->asg_choice, s1, s2);
  const uint32_t ncell = Gs[C->asg_choice].ncell;
  const uint32_t B = gv.B;
  int32_t* cnt = reinterpret_cast<int32_t*>(bm + B / 32u);  // difference array [B + 1]
  const uint32_t nidx = (S + WIN_IDX - 1u) / WIN_IDX;  // S <= 65536
  for (uint32_t j = tid; j < nidx; j += WIN_NT) sidx[j] = sorted[j * WIN_IDX];
  for (uint32_t b = tid; b <= B; b += WIN_NT) cnt[b] = 0;
  __syncthreads();
  GGMS_TRACE(18);
  // 1. bucket range of every k, as +1 / -1 in the difference array
  for (uint32_t i = tid; i < nk; i += WIN_NT) {
    const double q = ((double)krank[i] + 0.5) / (double)n;
    const double pos = q * (double)S;
    const double m = (double)z * sqrt((double)S * q * (1.0 - q)) + (double)z + 2.0;
    const double a = floor(pos - m), c = ceil(pos + m);
    const K klo = a < 0.0 ? (K)0 : sorted[min((uint32_t)a, S - 1u)];
    const K khi = c > (double)(S - 1u) ? key_max<K>() : sorted[(uint32_t)c];
    const uint32_t b0 = min(grid_eval<K>(gv, klo), B - 1u);
    const uint32_t b1 = min(grid_eval<K>(gv, khi), B - 1u);
    atomicAdd(&cnt[b0], 1);
    atomicAdd(&cnt[b1 + 1u], -1);
  }
  __syncthreads();
  GGMS_TRACE(19);
  // 2. buckets some k may hold, then their runs in bucket order (B / 32 <= 1024 words)
  coverage_bitmap(cnt, B, bm, red);
  const uint32_t nraw = bitmap_runs(bm, B / 32u, rs, re, WIN_MAXRAW, red);
  const uint32_t nraw2 = nraw;
  GGMS_TRACE(20);
  // 3. sample positions of the raw runs: [ss, se) = the sample keys whose
  //    bucket lies in the run (binary search over the sorted sample)
  if (tid < 2u * min(nraw, WIN_MAXRAW)) {
    const uint32_t j = tid >> 1;
    const uint32_t target = (tid & 1u) ? re[j] + 1u : rs[j];  // first sample with bucket >= target
    // coarse: the first indexed key with bucket >= target, in shared memory;
    // then within the WIN_IDX keys before it, in global memory
    uint32_t lo = 0, hi = nidx;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (min(grid_eval<K>(gv, sidx[mid]), B - 1u) >= target) hi = mid; else lo = mid + 1;
    }
    hi = min(lo * WIN_IDX, S);
    lo = lo ? (lo - 1u) * WIN_IDX + 1u : 0u;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (min(grid_eval<K>(gv, sorted[mid]), B - 1u) >= target) hi = mid; else lo = mid + 1;
    }
    if (tid & 1u) se[j] = lo; else ss[j] = lo;
  }
  __syncthreads();
  GGMS_TRACE(21);
  // 4. merge runs across gaps that hold under 1/256 of the sample; decide:
  //    at most L0_WIN runs holding at most a quarter of the sample
  if (tid == 0) {
    sw.on = 0;
    sw.R = 0;
    sw.cnt = 0;
    sw.tight = 0;
    uint32_t R = 0, hot = 0;
    if (nraw >= 1 && nraw <= WIN_MAXRAW && nraw2 == nraw) {
      uint32_t cs = rs[0], ce = re[0], cse = se[0], css = ss[0];
      bool ok = true;
      for (uint32_t i = 1; i <= nraw && ok; ++i) {
        if (i < nraw && (ss[i] - cse) * 256u < S) {
          ce = re[i];
          cse = se[i];
          continue;
        }
        if (R == L0_WIN) { ok = false; break; }
        sw.rb0[R] = cs;
        sw.rb1[R] = ce;
        hot += cse - css;
        ++R;
        if (i < nraw) { cs = rs[i]; ce = re[i]; css = ss[i]; cse = se[i]; }
      }
      if (ok && hot * 4u <= S) {
        sw.on = 1;
        sw.R = R;
        // buckets below the smallest key's or above the largest key's never
        // hold a key: a gap made only of those is empty
        const uint32_t bmin = min(grid_eval<K>(gv, (K)0), B - 1u);
        const uint32_t bmax = min(grid_eval<K>(gv, key_max<K>()), B - 1u);
        uint32_t ne = 0;
        for (uint32_t g = 0; g <= R; ++g) {
          // gap g lies between run g-1 and run g; gb0 > gb1 marks an empty gap
          const uint32_t g0 = g == 0 ? 0u : sw.rb1[g - 1] + 1u;
          const uint32_t g1 = g == R ? B : sw.rb0[g];  // one past the gap's last bucket
          const bool holds = g0 < g1 && g0 <= bmax && g1 > bmin;
          sw.gb0[g] = holds ? g0 : B;
          sw.gb1[g] = holds ? g1 - 1u : 0u;
          ne += holds ? 1u : 0u;
        }
        sw.cnt = ne >= 2u ? 1u : 0u;
        sw.tight = hot * 64u <= S ? 1u : 0u;
      }
    }
  }
  __syncthreads();
  GGMS_TRACE(22);
  // 5. key range of each run: [L(rb0), L(rb1 + 1) - 1], L(x) = smallest key with
  //    bucket >= x; the upper end is the largest key when no key reaches rb1 + 1
  if (sw.on && tid < 2u * sw.R) {
    const uint32_t r = tid >> 1;
    const bool upper = tid & 1u;
    K v;
    if (upper) {
      v = grid_last_key<K>(gv, ncell, sw.rb1[r]);
    } else {  // rb0 <= B - 1: the clamp to B - 1 does not change the answer
      v = sw.rb0[r] == 0u ? (K)0 : grid_inv<K>(gv, ncell, sw.rb0[r]);
    }
    if (upper) sw.hi[r] = v; else sw.lo[r] = v;
  }
  __syncthreads();
  if (tid == 0) {
    *W = sw;
    C->win_runs = sw.on ? sw.R : 0u;
  }
  GGMS_TRACE(23);
}

GGMS_END
