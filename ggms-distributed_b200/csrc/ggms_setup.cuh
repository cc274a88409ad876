// ggms_setup.cuh -- building the level-0 bucket assigner on the device.
//
// Sample -> sort -> a piecewise-linear model (Assigner, knots at sample
// quantiles) -> compiled into the Grid the two passes evaluate.  Everything
// after the sort runs in ONE kernel of one CTA (1024 threads); nothing goes
// back to the host.  The reference does the same job with a thrust sort of
// 1024 samples and 17 single-element cudaMemcpy calls to the host
// (DistributedSMOS/bucketMultiselect.cu:421-515).
#pragma once
#include "ggms_kernels.cuh"

GGMS_BEGIN

constexpr int SETUP_NT = 1024;

// ------------------------------------------------------------------ block helpers (1024 threads)
template <typename V>
__device__ __forceinline__ V warp_incl_scan(V v, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    V t = __shfl_up_sync(FULL, v, o);
    if ((int)lane >= o) v += t;
  }
  return v;
}

// Exclusive scan over the block (each thread one value); returns the exclusive
// prefix and writes the block total to *total.  `red` holds 33 V.
template <typename V>
__device__ V block_excl_scan(V v, V* red, V* total) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const V inc = warp_incl_scan(v, lane);
  if (lane == 31) red[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    V w = lane < (blockDim.x >> 5) ? red[lane] : (V)0;
    w = warp_incl_scan(w, lane);
    red[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  const V out = inc - v + (warp ? red[warp - 1] : (V)0);
  const V tot = red[(blockDim.x >> 5) - 1];
  __syncthreads();
  *total = tot;
  return out;
}

template <typename V>
__device__ V block_sum(V v, V* red) {
  V tot;
  block_excl_scan<V>(v, red, &tot);
  return tot;
}

// ------------------------------------------------------------------ PL model build
// Exclusive prefix max over the block in thread order (identity for thread 0).
template <typename V>
__device__ V block_excl_max(V v, V ident, V* red) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  V inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const V t = __shfl_up_sync(FULL, inc, o);
    if ((int)lane >= o) inc = max(inc, t);
  }
  V ex = __shfl_up_sync(FULL, inc, 1);
  if (lane == 0) ex = ident;
  if (lane == 31) red[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    V w = lane < (blockDim.x >> 5) ? red[lane] : ident;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const V t = __shfl_up_sync(FULL, w, o);
      if ((int)lane >= o) w = max(w, t);
    }
    red[lane] = w;
  }
  __syncthreads();
  const V out = warp ? max(ex, red[warp - 1]) : ex;
  __syncthreads();
  return out;
}

// Makes the bases Bs[0..m) of m knots strictly increasing and keeps them in
// [1, B-1] (m <= B - 1, m <= 2 * blockDim.x; all threads call it):
//   Bs[0] = 1;  Bs[t] = max(Bs[t], Bs[t-1] + 1)    (= t + max_{t' <= t} (Bs[t'] - t'))
//   Bs[m-1] = max(Bs[m-1], B - 1);  Bs[t] = max(1, min(Bs[t], B - 1 - (m - 1 - t)))
// The running maximum is one block-wide prefix max, two knots per thread.
__device__ void strict_bases(uint32_t* Bs, uint32_t m, uint32_t B, int32_t* red) {
  const uint32_t tid = threadIdx.x;
  int32_t d2[2] = {INT32_MIN, INT32_MIN};
  for (uint32_t k = 0; k < 2; ++k) {
    const uint32_t t = tid * 2 + k;
    if (t < m) d2[k] = ((t == 0) ? 1 : (int32_t)Bs[t]) - (int32_t)t;
  }
  d2[1] = max(d2[1], d2[0]);
  const int32_t dex = block_excl_max<int32_t>(d2[1], INT32_MIN, red);  // syncs: all reads done
  for (uint32_t k = 0; k < 2; ++k) {
    const uint32_t t = tid * 2 + k;
    if (t < m) {
      long long b = (long long)max(d2[k], dex) + (long long)t;
      if (t == m - 1) b = max(b, (long long)B - 1);
      const long long cap = (long long)B - 1 - ((long long)m - 1 - t);
      b = max(1LL, min(b, cap));
      if (m == 1) b = 1;
      Bs[t] = (uint32_t)b;
    }
  }
  __syncthreads();
}

struct BuildSmem {
  uint32_t jb[ASG_MAXM + 1];    // base of knot candidate j, non-decreasing in j
  uint32_t rend[ASG_MAXM + 1];  // last candidate of the run of equal knots starting at j
  uint32_t red_u[32];
  int32_t red_i[32];
};

// Builds a PL assigner from knot candidates: candidate j is sorted[q[j]] with
// target CDF cdf[j] (cdf[0] = 0, cdf[Mreq] = 1), j = 0..Mreq, Mreq <= ASG_MAXM.
// Runs of equal candidates (an atom of the sample) become one knot; an atom v
// gets a bucket of its own by an extra knot at v+1 whose base is the base at
// the run's end.  Bases are then made strictly increasing (distinct knots never
// share a bucket) and kept in [1, B-1].  Every step is a block-wide prefix
// scan over the candidates, two per thread; needs blockDim.x == SETUP_NT.
template <typename K>
__device__ void asg_build_from_knots(const K* sorted, const uint32_t* q, const float* cdf,
                                     uint32_t Mreq, uint32_t B, uint32_t kind, Assigner<K>* A) {
  __shared__ K XK[ASG_MAXM + 1];
  __shared__ K X[ASG_MAXM + 1];
  __shared__ uint32_t Bs[ASG_MAXM + 1];
  __shared__ BuildSmem bs;
  const uint32_t tid = threadIdx.x;
  const float span = (float)(B - 2u);
  // 1. candidate keys and bases; bases made non-decreasing by a prefix max
  uint32_t b2[2] = {0u, 0u};
  for (uint32_t k = 0; k < 2; ++k) {
    const uint32_t j = tid * 2 + k;
    if (j <= Mreq) {
      XK[j] = sorted[q[j]];
      const float f = fminf(fmaxf(cdf[j], 0.0f), 1.0f);
      uint32_t b = 1u + __float2uint_rn(f * span);
      if (j == 0) b = 1u;
      if (j == Mreq) b = B - 1u;
      b2[k] = b;
    }
  }
  b2[1] = max(b2[1], b2[0]);
  const uint32_t bex = block_excl_max<uint32_t>(b2[1], 0u, bs.red_u);  // also syncs XK
  // 2. run starts; every candidate learns its run's start by a prefix max
  bool start[2];
  uint32_t rs2[2] = {0u, 0u};
  for (uint32_t k = 0; k < 2; ++k) {
    const uint32_t j = tid * 2 + k;
    start[k] = j <= Mreq && (j == 0 || XK[j] != XK[j - 1]);
    if (j <= Mreq) bs.jb[j] = max(b2[k], bex);
    rs2[k] = start[k] ? j : 0u;
  }
  rs2[1] = max(rs2[1], rs2[0]);
  const uint32_t rsex = block_excl_max<uint32_t>(rs2[1], 0u, bs.red_u);
  for (uint32_t k = 0; k < 2; ++k) {
    const uint32_t j = tid * 2 + k;
    const bool end = j <= Mreq && (j == Mreq || XK[j + 1] != XK[j]);
    if (end) bs.rend[max(k ? rs2[1] : rs2[0], rsex)] = j;
  }
  __syncthreads();
  // 3. emit: a run start gives its knot, plus v+1 after an atom with room above
  uint32_t emit[2] = {0u, 0u};
  for (uint32_t k = 0; k < 2; ++k) {
    const uint32_t j = tid * 2 + k;
    if (start[k]) {
      const uint32_t e = bs.rend[j];
      emit[k] = (e > j && e < Mreq && (K)(XK[j] + 1) < XK[e + 1]) ? 2u : 1u;
    }
  }
  uint32_t m = 0;
  uint32_t at = block_excl_scan<uint32_t>(emit[0] + emit[1], bs.red_u, &m);
  for (uint32_t k = 0; k < 2; ++k) {
    const uint32_t j = tid * 2 + k;
    if (emit[k]) {
      X[at] = XK[j];
      Bs[at] = bs.jb[j];
      if (emit[k] == 2u) {
        X[at + 1] = (K)(XK[j] + 1);
        Bs[at + 1] = max(bs.jb[j] + 1u, bs.jb[bs.rend[j]]);
      }
      at += emit[k];
    }
  }
  __syncthreads();
  // 4. strictly increasing bases in [1, B-1]
  strict_bases(Bs, m, B, bs.red_i);
  const uint32_t M = m - 1;
  const K span_k = X[M] - X[0];
  const int csh = max(0, bitlen(span_k) - ASG_CELL_BITS);
  const uint32_t ncell = (uint32_t)(span_k >> csh) + 1u;
  if (tid == 0) {
    A->M = M;
    A->B = B;
    A->kind = kind;
    A->loss = 0.0f;
    A->csh = (uint32_t)csh;
    A->ncell = ncell;
  }
  for (uint32_t t = tid; t <= M; t += blockDim.x) {
    A->x[t] = X[t];
    A->base[t] = Bs[t];
    if (t < M) {
      const float db = (float)(Bs[t + 1] - Bs[t]);
      const float dx = key_to_float_rn((K)(X[t + 1] - X[t]));
      A->slope[t] = __fdiv_rn(db, dx);
    }
  }
  // cell index: idx[c] = last segment j <= M-1 whose knot is <= the cell's first key
  for (uint32_t c = tid; c < (uint32_t)ASG_NCELL; c += blockDim.x) {
    uint32_t j = 0;
    if (c < ncell && M > 0) {
      const K cstart = X[0] + ((K)c << csh);
      uint32_t lo = 0, hi = M - 1;  // largest j in [0, M-1] with X[j] <= cstart
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (X[mid] <= cstart) lo = mid; else hi = mid - 1;
      }
      j = lo;
    }
    A->idx[c] = (uint16_t)j;
  }
  __syncthreads();
}

// ------------------------------------------------------------------ grid compilation
// Resamples a monotone model (the PL assigner `a`) onto the grid; the heaviest
// bucket span is at least T (the smallest power of two >= 4x the mean span that
// leaves at most GRID_NSUB such cells) are split into sub-cells.  Writes the
// grid to `G` (global) and to the shared copies s1/s2.  All threads call it.
template <typename K>
struct CompileSmem {
  uint32_t bnd[GRID_NC1 + 1];   // bucket at each interior cell boundary
  uint32_t sub_base[GRID_NC1];  // first sub-cell entry of a split cell (0xFFFFFFFF: not split)
  uint32_t split_cell[GRID_SUBCAP / 2];  // split cells in order (each has >= 2 sub-cells)
  uint32_t split_base[GRID_SUBCAP / 2];
  uint32_t dev[GRID_NC1];       // max |PL - linear| at the knots inside a cell, in buckets
  uint32_t hist[33];
  uint32_t red[33];
  uint32_t thresh;
  uint32_t cap;
};

constexpr uint32_t GRID_DEV = 8;  // buckets of model deviation that make a cell worth splitting

// sub-cell bits of a split cell with bucket span sp under depth cap (cap <= sh1)
__device__ __forceinline__ uint32_t grid_sub_bits(uint32_t sp, int cap) {
  return (uint32_t)min(min(bitlen(sp), GRID_MAXSB), cap);
}

template <typename K>
__device__ GridView<K> grid_compile(const AsgView<K>& a, uint32_t B, uint32_t kind, Grid<K>* G,
                                    uint2* s1, uint2* s2, CompileSmem<K>& cs) {
  const uint32_t tid = threadIdx.x, NT = blockDim.x;
  const K KMAX = key_max<K>();
  const K lo = a.x[0];
  const K hi = a.x[a.M];
  const K span = (K)(hi - lo);
  const int sh1 = max(0, bitlen(span) - GRID_BITS1);
  const K w = (K)1 << sh1;
  const uint32_t nc = (uint32_t)(span >> sh1) + 1u;        // interior cells
  const bool has_lo = lo >= w;                              // room for a low tail cell
  // room for a high tail cell: KMAX - lo >= nc * w (computed without overflow)
  const bool has_hi = ((K)(KMAX - lo) >> sh1) >= (K)nc;
  const uint32_t first = has_lo ? 1u : 0u;
  const K origin = has_lo ? (K)(lo - w) : lo;
  K gmax = KMAX;
  if (has_hi) {
    const K top = (K)(lo + ((K)nc << sh1));                 // first key of the high tail cell
    gmax = ((K)(KMAX - top) >= (K)(w - 1)) ? (K)(top + (w - 1)) : KMAX;
  }
  const uint32_t ntot = first + nc + (has_hi ? 1u : 0u);
  for (uint32_t c = tid; c <= nc; c += NT) {
    uint32_t b;
    if (c < nc) b = asg_eval<K>(a, (K)(lo + ((K)c << sh1)));
    else b = asg_eval<K>(a, hi) + 1u;
    cs.bnd[c] = min(b, B - 1u);  // every grid entry stays a valid bucket
  }
  if (tid < 33) cs.hist[tid] = 0;
  for (uint32_t c = tid; c < nc; c += NT) cs.dev[c] = 0;
  __syncthreads();
  // Non-linearity of the model inside each cell: at every interior knot, the
  // distance (in buckets) between the model and the cell's linear interpolation.
  for (uint32_t k = 1 + tid; k < a.M; k += NT) {
    const K xk = a.x[k];
    const uint32_t c = (uint32_t)((K)(xk - lo) >> sh1);
    if (c >= nc) continue;
    const K off = (K)(xk - (K)(lo + ((K)c << sh1)));
    const float lin = (float)cs.bnd[c] + (float)(cs.bnd[c + 1] - cs.bnd[c]) *
                                             __fdiv_rn(key_to_float_rn(off), key_to_float_rn(w));
    const float d = fabsf((float)a.base[k] - lin);
    atomicMax(&cs.dev[c], (uint32_t)fminf(d, 1.0e9f));
  }
  __syncthreads();
  // Split the cells where the model bends (deviation >= GRID_DEV buckets) so
  // that a sub-cell spans about one bucket: a cell of bucket span sp gets
  // 2^min(bitlen(sp), cap) sub-cells.  cap is the largest depth (<= GRID_MAXSB)
  // whose total fits GRID_SUBCAP entries; if even depth 1 does not fit, only the
  // cells with bitlen(sp) >= t are split (at depth 1), t the smallest that fits.
  auto wants_split = [&](uint32_t c) -> bool {
    const uint32_t sp = cs.bnd[c + 1] - cs.bnd[c];
    return sp >= 4u && sh1 >= 1 && cs.dev[c] >= GRID_DEV;
  };
  for (uint32_t c = tid; c < nc; c += NT)
    if (wants_split(c)) atomicAdd(&cs.hist[bitlen(cs.bnd[c + 1] - cs.bnd[c])], 1u);
  __syncthreads();
  if (tid == 0) {
    uint32_t cap = 0, t = 3;
    for (int d = min(GRID_MAXSB, sh1); d >= 1 && cap == 0; --d) {
      uint32_t cost = 0;
      for (int k = 3; k <= 32; ++k) cost += cs.hist[k] << (uint32_t)min(k, d);
      if (cost <= (uint32_t)GRID_SUBCAP) cap = (uint32_t)d;
    }
    if (cap == 0 && sh1 >= 1) {  // too many heavy cells: depth 1 for the heaviest only
      uint32_t cost = 0;
      t = 33;
      for (int k = 32; k >= 3; --k) {
        if (cost + (cs.hist[k] << 1) > (uint32_t)GRID_SUBCAP) break;
        cost += cs.hist[k] << 1;
        t = (uint32_t)k;
      }
      cap = 1;
    }
    cs.thresh = t;
    cs.cap = cap;
  }
  __syncthreads();
  const uint32_t thr = cs.thresh, cap = cs.cap;
  // sub-table bases: prefix over the split cells' sizes in cell order (2 cells per thread)
  uint32_t sz[2] = {0, 0};
  for (uint32_t k = 0; k < 2; ++k) {
    const uint32_t c = tid * 2 + k;
    if (c < nc) {
      const uint32_t sp = cs.bnd[c + 1] - cs.bnd[c];
      if (cap && wants_split(c) && (uint32_t)bitlen(sp) >= thr) sz[k] = 1u << grid_sub_bits(sp, cap);
    }
  }
  uint32_t total = 0;
  const uint32_t pre = block_excl_scan<uint32_t>(sz[0] + sz[1], cs.red, &total);
  uint32_t nsplit_tot = 0;
  const uint32_t spre = block_excl_scan<uint32_t>((sz[0] ? 1u : 0u) + (sz[1] ? 1u : 0u), cs.red, &nsplit_tot);
  {
    uint32_t base = pre, si = spre;
    for (uint32_t k = 0; k < 2; ++k) {
      const uint32_t c = tid * 2 + k;
      if (c < nc) {
        if (sz[k]) {
          cs.sub_base[c] = base;
          cs.split_cell[si] = c;
          cs.split_base[si] = base;
          ++si;
          base += sz[k];
        } else {
          cs.sub_base[c] = 0xFFFFFFFFu;
        }
      }
    }
  }
  __syncthreads();
  for (uint32_t c = tid; c < ntot; c += NT) {
    uint2 e;
    if (c < first) {
      e = make_uint2(0u, 0u);                                 // low tail: bucket 0
    } else if (c >= first + nc) {
      e = make_uint2(B - 1u, B - 1u);                         // high tail: bucket B-1
    } else {
      const uint32_t i = c - first;
      const uint32_t sb0 = cs.sub_base[i];
      if (sb0 != 0xFFFFFFFFu) {
        const uint32_t sp = cs.bnd[i + 1] - cs.bnd[i];
        e = make_uint2(GRID_SPLIT | (grid_sub_bits(sp, (int)cap) << 16), sb0);
      } else {
        e = make_uint2(cs.bnd[i], cs.bnd[i + 1]);
      }
    }
    s1[c] = e;
    G->t1[c] = e;
  }
  // sub-cell entries
  for (uint32_t i = tid; i < total; i += NT) {
    uint32_t lo_i = 0, hi_i = nsplit_tot - 1;  // last split cell whose base <= i
    while (lo_i < hi_i) {
      const uint32_t m = (lo_i + hi_i + 1) >> 1;
      if (cs.split_base[m] <= i) lo_i = m; else hi_i = m - 1;
    }
    const uint32_t c = cs.split_cell[lo_i];
    const uint32_t s = i - cs.split_base[lo_i];
    const uint32_t sb = grid_sub_bits(cs.bnd[c + 1] - cs.bnd[c], (int)cap);
    const int shs = sh1 - (int)sb;
    const K cell_lo = (K)(lo + ((K)c << sh1));
    const K room = (K)(hi - cell_lo);  // sub-boundaries past hi (last cell only) take the cell's end
    auto bnd_at = [&](uint32_t q) -> uint32_t {
      if (q == (1u << sb)) return cs.bnd[c + 1];
      const K off = (K)q << shs;
      return off > room ? cs.bnd[c + 1] : min(asg_eval<K>(a, (K)(cell_lo + off)), cs.bnd[c + 1]);
    };
    const uint2 e = make_uint2(bnd_at(s), bnd_at(s + 1));
    s2[i] = e;
    G->t2[i] = e;
  }
  if (tid == 0) {
    G->origin = origin;
    G->gmax = gmax;
    G->sh1 = (uint32_t)sh1;
    G->nsubent = total;
    G->B = B;
    G->ncell = ntot;
    G->nsplit = nsplit_tot;
    G->kind = kind;
    G->loss = 0.0f;
  }
  __syncthreads();
  GridView<K> v;
  v.t1 = s1; v.t2 = s2; v.origin = origin; v.gmax = gmax;
  v.sh1 = (uint32_t)sh1; v.B = B;
  return v;
}

// ------------------------------------------------------------------ interval bitmaps
// Sets bits [b0, b1] of a bitmap in shared memory (concurrent callers OK).
__device__ __forceinline__ void bits_mark(uint32_t* bm, uint32_t b0, uint32_t b1) {
  const uint32_t w0 = b0 >> 5, w1 = b1 >> 5;
  const uint32_t lo = ~0u << (b0 & 31);
  const uint32_t hi = (b1 & 31) == 31u ? ~0u : ((2u << (b1 & 31)) - 1u);
  if (w0 == w1) {
    atomicOr(&bm[w0], lo & hi);
    return;
  }
  atomicOr(&bm[w0], lo);
  for (uint32_t w = w0 + 1u; w < w1; ++w) atomicOr(&bm[w], ~0u);
  atomicOr(&bm[w1], hi);
}

// Coverage of intervals given as a difference array cnt[0..nb] (+1 at each
// interval's first bin, -1 one past its last; nb a multiple of blockDim.x):
// bm gets one bit per bin, set where the coverage is > 0.  Warp w scans bins
// [w * nb / nwarps, (w + 1) * nb / nwarps) row by row (32 bins per row, one per
// lane: no bank conflicts).  All threads call it.
__device__ void coverage_bitmap(const int32_t* cnt, uint32_t nb, uint32_t* bm, uint32_t* red) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t per = nb / nw, base = warp * per;
  int32_t part = 0;
  for (uint32_t r = 0; r < per; r += 32) part += cnt[base + r + lane];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(FULL, part, o);
  uint32_t tot = 0;
  // block-exclusive prefix of the warp sums (lane 0 of warp w contributes part_w)
  int32_t run = (int32_t)block_excl_scan<uint32_t>(lane == 0 ? (uint32_t)part : 0u, red, &tot);
  run = __shfl_sync(FULL, run, 0);
  for (uint32_t r = 0; r < per; r += 32) {
    int32_t v = cnt[base + r + lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t t = __shfl_up_sync(FULL, v, o);
      if ((int)lane >= o) v += t;
    }
    const uint32_t bits = __ballot_sync(FULL, run + v > 0);
    if (lane == 0) bm[(base + r) >> 5] = bits;
    run += __shfl_sync(FULL, v, 31);
  }
  __syncthreads();
}

// Maximal runs of set bits of a bitmap of `words` words (<= blockDim.x), in
// order: run j is [rs[j], re[j]] for j < min(total, cap).  Returns the number
// of runs.  All threads call it.
__device__ uint32_t bitmap_runs(const uint32_t* bm, uint32_t words, uint32_t* rs, uint32_t* re,
                                uint32_t cap, uint32_t* red) {
  const uint32_t i = threadIdx.x;
  uint32_t st = 0, en = 0;
  if (i < words) {
    const uint32_t w = bm[i];
    const uint32_t prev_top = i ? bm[i - 1] >> 31 : 0u;
    const uint32_t next_low = i + 1u < words ? bm[i + 1u] & 1u : 0u;
    st = w & ~((w << 1) | prev_top);
    en = w & ~((w >> 1) | (next_low << 31));
  }
  uint32_t total = 0, total2 = 0;
  uint32_t a = block_excl_scan<uint32_t>((uint32_t)__popc(st), red, &total);
  uint32_t b = block_excl_scan<uint32_t>((uint32_t)__popc(en), red, &total2);
  while (st) {
    const uint32_t bit = __ffs(st) - 1u;
    if (a < cap) rs[a] = i * 32u + bit;
    ++a;
    st &= st - 1u;
  }
  while (en) {
    const uint32_t bit = __ffs(en) - 1u;
    if (b < cap) re[b] = i * 32u + bit;
    ++b;
    en &= en - 1u;
  }
  __syncthreads();
  return total;
}

// ------------------------------------------------------------------ bucket focus
// A monotone piecewise-linear map of CDF space onto itself, w(0) = 0,
// w(1) = 1: a learned model places bucket boundaries at w(F(key)) instead of
// F(key).  With the ks clustered, the CDF ranges that can hold a k (the same
// windows PASS 1 uses) get most of the buckets and the gaps between them the
// rest, so the buckets that hold a k are far smaller and the candidates far
// fewer.  Identity (n = 2 points) when the ks are spread out.
constexpr uint32_t WARP_PTS = 2 * 4 + 2;   // two breakpoints per run (<= 4 runs) + the ends
constexpr uint32_t FOCUS_BINS = 4096;     // resolution of the windows in CDF space
constexpr float FOCUS_GAPS = 0.125f;      // share of the buckets for the gaps between runs

struct Warp {
  uint32_t n;              // breakpoints, 2..WARP_PTS
  float p[WARP_PTS];       // CDF values, increasing from 0 to 1
  float w[WARP_PTS];       // their images, increasing from 0 to 1
};

__device__ __forceinline__ float warp_fwd(const Warp& W, float p) {
  p = fminf(fmaxf(p, 0.0f), 1.0f);
  for (uint32_t i = 1; i < W.n; ++i)
    if (p <= W.p[i] || i + 1 == W.n) {
      const float d = W.p[i] - W.p[i - 1];
      return d > 0.0f ? W.w[i - 1] + (W.w[i] - W.w[i - 1]) * __fdiv_rn(p - W.p[i - 1], d) : W.w[i];
    }
  return 1.0f;
}
__device__ __forceinline__ float warp_inv(const Warp& W, float y) {
  y = fminf(fmaxf(y, 0.0f), 1.0f);
  for (uint32_t i = 1; i < W.n; ++i)
    if (y <= W.w[i] || i + 1 == W.n) {
      const float d = W.w[i] - W.w[i - 1];
      return d > 0.0f ? W.p[i - 1] + (W.p[i] - W.p[i - 1]) * __fdiv_rn(y - W.w[i - 1], d) : W.p[i];
    }
  return 1.0f;
}

// Builds the warp from the ks (ascending ranks krank[0..nk) of n keys) and the
// sample size S.  The window of a k in CDF space is [pos - m, pos + m] / S with
// pos = S (r + 1/2) / n and m = z sqrt(S q (1 - q)) + z + 2 (the PASS 1 window
// rule); windows are rasterised onto a bitmap of FOCUS_BINS bins, merged
// across gaps narrower than FOCUS_BINS / 256 bins, and used when they form at
// most `maxruns` runs covering at most a quarter of the CDF.  All threads call
// it (blockDim.x >= FOCUS_BINS / 32); scratch holds FOCUS_BINS / 32 + 128
// words of shared memory.
__device__ void build_warp(const uint32_t* __restrict__ krank, uint32_t nk, uint64_t n, uint32_t S,
                           float z, uint32_t maxruns, uint32_t* scratch, uint32_t* red, Warp* out) {
  constexpr uint32_t WORDS = FOCUS_BINS / 32u, CAP = 64;
  uint32_t* bm = scratch;              // [WORDS] covered bins
  uint32_t* rs = scratch + WORDS;      // [CAP] raw run starts
  uint32_t* re = rs + CAP;             // [CAP] raw run ends
  const uint32_t tid = threadIdx.x, NT = blockDim.x;
  for (uint32_t w = tid; w < WORDS; w += NT) bm[w] = 0u;
  __syncthreads();
  for (uint32_t i = tid; i < nk; i += NT) {
    const double q = ((double)krank[i] + 0.5) / (double)n;
    const double m = (double)z * sqrt((double)S * q * (1.0 - q)) + (double)z + 2.0;
    const double a = q - m / (double)S, c = q + m / (double)S;
    const uint32_t b0 = a <= 0.0 ? 0u : min((uint32_t)(a * FOCUS_BINS), FOCUS_BINS - 1u);
    const uint32_t b1 = c >= 1.0 ? FOCUS_BINS - 1u : min((uint32_t)(c * FOCUS_BINS), FOCUS_BINS - 1u);
    bits_mark(bm, b0, b1);
  }
  __syncthreads();
  const uint32_t nraw = bitmap_runs(bm, WORDS, rs, re, CAP, red);
  if (tid == 0) {
    // merge runs across narrow gaps
    constexpr uint32_t MERGE = FOCUS_BINS / 256u;
    uint32_t frs[4], fre[4], R = 0, cov = 0;
    bool ok = nraw >= 1u && nraw <= CAP;
    for (uint32_t j = 0; j < nraw && ok; ++j) {
      if (R > 0 && rs[j] - fre[R - 1] - 1u < MERGE) {
        fre[R - 1] = re[j];
      } else if (R < 4u && R < maxruns) {
        frs[R] = rs[j];
        fre[R] = re[j];
        ++R;
      } else {
        ok = false;
      }
    }
    for (uint32_t r = 0; r < R; ++r) cov += fre[r] - frs[r] + 1u;
    Warp W;
    W.n = 2;
    W.p[0] = 0.0f; W.w[0] = 0.0f;
    W.p[1] = 1.0f; W.w[1] = 1.0f;
    if (ok && R > 0 && cov <= FOCUS_BINS / 4u) {
      const float P = (float)cov / (float)FOCUS_BINS;  // CDF mass of the runs
      const float gap_share = (P < 1.0f) ? FOCUS_GAPS : 0.0f;
      const float run_slope = (1.0f - gap_share) / P, gap_slope = gap_share / (1.0f - P);
      uint32_t k = 0;
      float pp = 0.0f, ww = 0.0f;
      W.p[k] = 0.0f; W.w[k] = 0.0f; ++k;
      for (uint32_t r = 0; r < R; ++r) {
        const float a = (float)frs[r] / (float)FOCUS_BINS, c = (float)(fre[r] + 1u) / (float)FOCUS_BINS;
        if (a > pp) {  // gap before run r
          ww += (a - pp) * gap_slope;
          pp = a;
          W.p[k] = pp; W.w[k] = fminf(ww, 1.0f); ++k;
        }
        ww += (c - pp) * run_slope;
        pp = c;
        W.p[k] = pp; W.w[k] = fminf(ww, 1.0f); ++k;
      }
      if (pp < 1.0f) { W.p[k] = 1.0f; W.w[k] = 1.0f; ++k; }
      W.w[k - 1] = 1.0f;
      W.n = k;
    }
    *out = W;
  }
  __syncthreads();
}

// Occupancy of the grid's buckets on the (sorted) sample, over 256 groups of
// buckets: max / mean.
// At most GRID_MEASURE_N samples are used (a strided subsample of the sorted
// sample, still sorted): 16 per group on average, enough to see imbalance
// against the bound (3.0: a group holding three times its share; a model that
// fits the sample exactly reads about 1.8 from the sampling noise alone), and
// all of a thread's samples are loaded at once.
constexpr uint32_t GRID_MEASURE_N = 4096;

template <typename K>
__device__ float grid_measure(const GridView<K>& g, const K* sorted_all, uint32_t S_all, uint32_t* hist256,
                              const Warp* wp = nullptr) {
  const uint32_t stride = S_all > GRID_MEASURE_N ? S_all / GRID_MEASURE_N : 1u;
  const uint32_t S = S_all / stride;
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) hist256[i] = 0;
  __syncthreads();
  // coalesced loads, eight in flight per thread; the sample is sorted, so the
  // 32 lanes of a warp usually share a group: one add per warp then
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t NTh = blockDim.x;
  for (uint32_t base = 0; base < S; base += 8 * NTh) {
    K v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t i = base + u * NTh + threadIdx.x;
      v[u] = i < S ? sorted_all[(size_t)i * stride] : (K)0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t i = base + u * NTh + threadIdx.x;
      const bool ok = i < S;
      uint32_t grp = 0xFFFFFFFFu;
      if (ok) {
        const uint32_t b = grid_eval<K>(g, v[u]);
        if (wp && wp->n > 2u) {  // a focused model: measure in the CDF space before the warp
          const float y = ((float)b - 0.5f) / (float)(g.B - 2u);
          grp = min((uint32_t)(warp_inv(*wp, y) * 256.0f), 255u);
        } else {
          grp = (uint32_t)(((uint64_t)b * 256u) / g.B);
        }
      }
      const uint32_t g0 = __shfl_sync(FULL, grp, 0);
      const uint32_t okm = __ballot_sync(FULL, ok);
      if (__all_sync(FULL, !ok || grp == g0)) {
        if (lane == 0 && okm) atomicAdd(&hist256[g0], (uint32_t)__popc(okm));
      } else if (ok) {
        atomicAdd(&hist256[grp], 1u);
      }
    }
  }
  __syncthreads();
  // the largest group: 8 warps reduce 32 counts each, then every thread reads the 8
  __shared__ uint32_t wmax[8];
  if (threadIdx.x < 256) {
    uint32_t m = hist256[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(FULL, m, o));
    if (lane == 0) wmax[threadIdx.x >> 5] = m;
  }
  __syncthreads();
  uint32_t mx = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) mx = max(mx, wmax[w]);
  __syncthreads();
  return (float)mx / ((float)S / 256.0f);
}

// Copy a PL assigner (global) into shared memory.
template <typename K>
struct AsgCopy {
  K x[ASG_MAXM + 1];
  uint32_t base[ASG_MAXM + 1];
  float slope[ASG_MAXM];
  uint16_t idx[ASG_NCELL];
};

template <typename K>
__device__ AsgView<K> asg_copy(const Assigner<K>* A, AsgCopy<K>& c) {
  const uint32_t M = A->M;
  for (uint32_t i = threadIdx.x; i <= M; i += blockDim.x) {
    c.x[i] = A->x[i];
    c.base[i] = A->base[i];
    if (i < M) c.slope[i] = A->slope[i];
  }
  for (uint32_t i = threadIdx.x; i < A->ncell; i += blockDim.x) c.idx[i] = A->idx[i];
  __syncthreads();
  AsgView<K> v;
  v.x = c.x; v.base = c.base; v.slope = c.slope; v.idx = c.idx;
  v.M = M; v.B = A->B; v.csh = A->csh;
  return v;
}

template <typename K>
struct SetupSmem {
  AsgCopy<K> asg;
  CompileSmem<K> cs;
  uint2 s1[GRID_T1];
  uint2 s2[GRID_SUBCAP];
  uint32_t hist256[256];
};

// The reference's pivot rule (bucketMultiselect.cu:421-515, sizeOfSample = 1024,
// numPivots = 17, endOffset = 22, pivotOffset = (1024 - 44) / 14 = 70):
// pivots {min, s[21], s[21 + 70(i-1)] for i = 2..14, s[1001], max}, every
// segment gets the same number of buckets.  The global min and max (a full
// minmax pass in the reference) are replaced by the sample's extremes plus an
// open tail bucket at each end.  For other sample sizes the offsets scale.
// One CTA: pivots -> PL assigner A -> grid G -> occupancy on the sample.
template <typename K>
__global__ __launch_bounds__(SETUP_NT) void setup_sampled(const K* __restrict__ sorted, uint32_t S,
                                                         uint32_t B, Assigner<K>* A, Grid<K>* G) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem[];
  SetupSmem<K>& sm = *reinterpret_cast<SetupSmem<K>*>(smem);
  __shared__ uint32_t q[17];
  __shared__ float cdf[17];
  GGMS_TRACE(3);
  if (threadIdx.x == 0) {
    const uint32_t end_off = max(1u, (22u * S) / 1024u);
    const uint32_t piv_off = (S - 2u * end_off) / 14u;
    q[0] = 0;
    q[1] = end_off - 1u;
    for (uint32_t i = 2; i <= 14; ++i) q[i] = piv_off * (i - 1u) + end_off - 1u;
    q[15] = S - end_off - 1u;
    q[16] = S - 1u;
    for (int i = 0; i <= 16; ++i) cdf[i] = (float)i / 16.0f;
  }
  __syncthreads();
  asg_build_from_knots<K>(sorted, q, cdf, 16u, B, GGMS_ASSIGNER_SAMPLED, A);
  __syncthreads();
  const AsgView<K> av = asg_copy<K>(A, sm.asg);
  const GridView<K> gv = grid_compile<K>(av, B, GGMS_ASSIGNER_SAMPLED, G, sm.s1, sm.s2, sm.cs);
  const float qv = grid_measure<K>(gv, sorted, S, sm.hist256);
  if (threadIdx.x == 0) G->quality = qv;
  GGMS_TRACE(4);
}

GGMS_END
