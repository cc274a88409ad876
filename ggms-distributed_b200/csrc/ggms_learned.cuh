// ggms_learned.cuh -- learned level-0 bucket assigners, trained on the GPU.
//
// The reference places buckets with 17 sampled pivots and one linear slope per
// pivot interval (DistributedSMOS/bucketMultiselect.cu:421-515); data whose
// density changes inside an interval (mixtures, heavy tails) fills some buckets
// far more than others, and the reference's iterativeSMOS then needs many
// refinement rounds (DistributedSMOS/iterativeSMOS.cu:1348, outputfile.txt:7-71).
// Here a monotone CDF model is fitted to key/rank samples the selector draws
// itself, then compiled into the same piecewise-linear Assigner format the
// passes evaluate.  The model only places buckets: the counting and compaction
// passes still decide every answer exactly.
//
// PL-CDF model (M <= 1024 segments between knots at sample quantiles):
//   delta_j = softplus(theta_j) > 0,  P_j = sum_{t<j} delta_t,  D = sum_t delta_t
//   F(s) = (P_j + u(s) * delta_j) / D   for s in segment j, u = (s - x_j)/(x_{j+1} - x_j)
//   loss = 1/S * sum_i (F(s_i) - y_i)^2,  y_i = (i + 0.5) / S  (sorted sample)
// The loss and its gradient depend on the data only through six per-segment
// sums (n, sum u, sum u^2, sum y, sum y u, sum y^2), gathered once by
// pl_stats; every optimizer step is then O(M) work in one warp (pl_train).
//
// MLP-CDF model (1-32-32-1, monotone): see ggms_mlp.cuh.
#pragma once
#include "ggms_setup.cuh"

GGMS_BEGIN

constexpr int PL_M = 1024;       // segments of the learned PL model
constexpr int MLP_H = 32;        // hidden width of the MLP model
constexpr int MLP_NPARAM = 1153; // 32 + 32 + 32*32 + 32 + 32 + 1

struct PLStats {                 // per segment, in double for a stable sum
  double n, su, su2, sy, syu, sy2;
};

struct LearnState {
  float theta[PL_M];             // trained PL parameters
  float grad[PL_M];              // gradient at the trained parameters
  float cdf[PL_M + 1];           // trained CDF at the knots (MLP: its values at the knots)
  float loss_init;               // loss before training
  float loss;                    // loss after training
  float imbalance;               // max/mean of the compiled model on the sample
  uint32_t M;                    // segments actually used
  uint32_t steps;
  uint32_t choice;               // 1 learned accepted, 0 fell back to sampled
  uint32_t focus_points;         // breakpoints of the bucket focus (2: none)
  uint32_t pad[1];
  Warp warp;                     // the bucket focus (setup_pl_knots builds it, the bases use it)
  PLStats st[PL_M];              // per-segment statistics (pl_stats_grid -> training)
  // MLP parameters (see ggms_mlp.cuh)
  float mlp_params[MLP_NPARAM + 3];
  float mlp_loss;
};

__device__ __forceinline__ float softplusf(float x) {
  return x > 20.0f ? x : log1pf(expf(x));
}
__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + expf(-x)); }

// ------------------------------------------------------------------ statistics
// Per-segment sufficient statistics of the sorted sample, one warp per
// segment over many CTAs: the lanes stride the segment's samples (coalesced),
// each lane sums in sample order and the warp reduces in a fixed shape
// (deterministic).  A segment's first sample is found by one search per
// bound, first over every PL_IDX-th sample key kept in shared memory, then
// over the PL_IDX keys between two of them.  Grid: ceil(PL_M / 32) CTAs of
// 1024 threads; segments past A->M return.
constexpr uint32_t PL_IDX = 64;

template <typename K>
__global__ __launch_bounds__(1024) void pl_stats_grid(const K* __restrict__ sorted, uint32_t S,
                                                     const Assigner<K>* __restrict__ A, LearnState* L) {
  pdl_entry();
  __shared__ K sidx[65536u / PL_IDX];
  GGMS_TRACE(7);
  const uint32_t M = A->M;
  const uint32_t nidx = (S + PL_IDX - 1u) / PL_IDX;  // S <= 65536
  for (uint32_t j = threadIdx.x; j < nidx; j += blockDim.x) sidx[j] = sorted[j * PL_IDX];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= M) return;
  uint32_t bound = S;  // lane 0: first sample of segment j; lane 1: of segment j + 1
  if (lane < 2u && j + lane < M) {
    const K v = A->x[j + lane];
    uint32_t a = 0, b = nidx;  // first indexed key >= v
    while (a < b) { const uint32_t m = (a + b) >> 1; if (sidx[m] < v) a = m + 1; else b = m; }
    uint32_t hi = min(a * PL_IDX, S), lo = a ? (a - 1u) * PL_IDX + 1u : 0u;
    while (lo < hi) { const uint32_t m = (lo + hi) >> 1; if (sorted[m] < v) lo = m + 1; else hi = m; }
    bound = lo;
  }
  const uint32_t i0 = __shfl_sync(FULL, bound, 0), i1 = __shfl_sync(FULL, bound, 1);
  const K xj = A->x[j], xn = A->x[j + 1];
  const float width = key_to_float_rn((K)(xn - xj));
  double n = 0, su = 0, su2 = 0, sy = 0, syu = 0, sy2 = 0;
  for (uint32_t i = i0 + lane; i < i1; i += 32) {
    const float u = fminf(__fdiv_rn(key_to_float_rn((K)(sorted[i] - xj)), width), 1.0f);
    const double y = ((double)i + 0.5) / (double)S;
    n += 1.0; su += u; su2 += (double)u * u; sy += y; syu += y * u; sy2 += y * y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n += __shfl_xor_sync(FULL, n, o);
    su += __shfl_xor_sync(FULL, su, o);
    su2 += __shfl_xor_sync(FULL, su2, o);
    sy += __shfl_xor_sync(FULL, sy, o);
    syu += __shfl_xor_sync(FULL, syu, o);
    sy2 += __shfl_xor_sync(FULL, sy2, o);
  }
  if (lane == 0) L->st[j] = PLStats{n, su, su2, sy, syu, sy2};
  GGMS_TRACE(8);
}

// The statistics into shared memory for training (all threads call it).
__device__ __forceinline__ void pl_stats_load(const LearnState* L, uint32_t M, PLStats* st) {
  const double* src = reinterpret_cast<const double*>(L->st);
  double* dst = reinterpret_cast<double*>(st);
  for (uint32_t i = threadIdx.x; i < 6u * M; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// ------------------------------------------------------------------ forward / backward
// Run by the first PL_NT threads, synchronised with named barrier 1 (with
// PL_NT == blockDim.x that is the whole CTA).  Thread j owns segment j.
constexpr int PL_NT = PL_M;
__device__ __forceinline__ void bar_pl() { asm volatile("bar.sync 1, %0;" ::"n"(PL_NT) : "memory"); }

// Cross-warp partials of pl_fb and their combinations (made by warp 0).
struct PLRed {
  double a[PL_NT / 32], b[PL_NT / 32], c[PL_NT / 32], e[PL_NT / 32];
  double pa[PL_NT / 32], pb[PL_NT / 32];  // exclusive prefixes over the warps
  double ta, tb, tc, te;                  // totals
};

// Warp 0: exclusive prefix of x[0..32) into pre[], the total into *tot.
__device__ __forceinline__ void warp0_prefix(const double* x, double* pre, double* tot, uint32_t lane) {
  const double v = x[lane];
  const double inc = warp_incl_scan(v, lane);
  pre[lane] = inc - v;
  if (lane == 31) *tot = inc;
}
__device__ __forceinline__ void warp0_sum(const double* x, double* tot, uint32_t lane) {
  double v = x[lane];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  if (lane == 0) *tot = v;
}

// Returns the loss; *g = d loss / d theta_j; cdf_out (if given) gets P_j / D and 1 at M.
// Four named barriers: each cross-warp sum or prefix is formed once, by warp 0.
__device__ float pl_fb(float theta, const PLStats* st, uint32_t M, double S, PLRed& red, float* g,
                       float* cdf_out) {
  static_assert(PL_NT == 1024, "warp 0 combines exactly 32 warp partials");
  const uint32_t j = threadIdx.x, lane = j & 31, warp = j >> 5;
  const bool act = j < M;
  const double d = act ? (double)softplusf(theta) : 0.0;
  // P_j = sum_{t<j} d_t, D = sum d
  const double inc = warp_incl_scan(d, lane);
  if (lane == 31) red.a[warp] = inc;
  bar_pl();
  if (warp == 0) warp0_prefix(red.a, red.pa, &red.ta, lane);
  bar_pl();
  const double P = inc - d + red.pa[warp], D = red.ta;
  const double invD = 1.0 / D;
  double R = 0, U = 0, Qc = 0, Lc = 0;
  if (act) {
    const PLStats s = st[j];
    const double p = P * invD, dd = d * invD;
    // F_i = p + dd u_i ;  r_i = F_i - y_i
    R = s.n * p + dd * s.su - s.sy;
    U = p * s.su + dd * s.su2 - s.syu;
    const double sF2 = s.n * p * p + 2.0 * p * dd * s.su + dd * dd * s.su2;
    const double sFy = p * s.sy + dd * s.syu;
    Qc = sF2 - sFy;
    Lc = sF2 - 2.0 * sFy + s.sy2;
    if (cdf_out) cdf_out[j] = (float)p;
  }
  // suffix of R and totals of Qc, Lc
  const double rin = warp_incl_scan(R, lane);
  double q = Qc, l = Lc;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    q += __shfl_xor_sync(FULL, q, o);
    l += __shfl_xor_sync(FULL, l, o);
  }
  if (lane == 31) red.b[warp] = rin;
  if (lane == 0) { red.c[warp] = q; red.e[warp] = l; }
  bar_pl();
  if (warp == 0) {
    warp0_prefix(red.b, red.pb, &red.tb, lane);
    warp0_sum(red.c, &red.tc, lane);
    warp0_sum(red.e, &red.te, lane);
  }
  bar_pl();
  const double before = rin + red.pb[warp], Rt = red.tb, Q = red.tc, L = red.te;
  // dF_i/d delta_t = (1{t < j_i} + u_i 1{t = j_i} - F_i) / D
  const double after = Rt - before;
  if (act) *g = (float)((2.0 / (S * D)) * (after + U - Q) * (double)sigmoidf_(theta));
  else *g = 0.0f;
  if (cdf_out && j == 0) cdf_out[M] = 1.0f;
  return (float)(L / S);
}

// Adam on theta (thread j owns theta_j).  Returns the best loss seen.  Every
// evaluation writes its CDF at the knots, alternating between cdf_out and
// cdf_alt so that the best one is never overwritten: no final evaluation is
// needed; thread 0 stores 1 in *in_alt when the best CDF is in cdf_alt.
__device__ float pl_train_block(const PLStats* st, uint32_t M, uint32_t S, uint32_t steps, float lr,
                                PLRed& red, float* cdf_out, float* cdf_alt, uint32_t* in_alt,
                                float* loss0_out, float* theta_out, float* grad_out) {
  // start from the sample's own CDF: increments proportional to each segment's
  // sample count (for knots at uniform quantiles, all 1: softplus^-1(1))
  float theta;
  {
    const float c = threadIdx.x < M ? (float)st[threadIdx.x].n : 0.0f;
    const float delta = fmaxf(c * (float)M / (float)S, 1.0e-4f);
    theta = delta > 20.0f ? delta : logf(expm1f(delta));
  }
  float m1 = 0.0f, m2 = 0.0f, g = 0.0f;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float b1t = 1.0f, b2t = 1.0f;
  float loss = pl_fb(theta, st, M, (double)S, red, &g, cdf_out);
  if (loss0_out && threadIdx.x == 0) *loss0_out = loss;
  // keep the best parameters seen: the initialisation is already close to the
  // optimum, so a step can overshoot; the result never loses to the init
  float best = loss, best_theta = theta, best_g = g;
  bool alt = false;  // the best CDF is in cdf_alt
  for (uint32_t it = 0; it < steps; ++it) {
    b1t *= b1;
    b2t *= b2;
    m1 = b1 * m1 + (1.0f - b1) * g;
    m2 = b2 * m2 + (1.0f - b2) * g * g;
    theta -= lr * (m1 / (1.0f - b1t)) / (sqrtf(m2 / (1.0f - b2t)) + eps);
    loss = pl_fb(theta, st, M, (double)S, red, &g, alt ? cdf_out : cdf_alt);
    if (loss < best) {  // the loss is block-uniform: every thread takes the same branch
      best = loss;
      best_theta = theta;
      best_g = g;
      alt = !alt;
    }
  }
  if (theta_out && threadIdx.x < M) theta_out[threadIdx.x] = best_theta;
  if (grad_out && threadIdx.x < M) grad_out[threadIdx.x] = best_g;
  if (threadIdx.x == 0) *in_alt = alt ? 1u : 0u;
  return best;
}

// New bases (strictly increasing) and slopes of a PL assigner from CDF values
// at its knots.  All threads call it.
template <typename K>
__device__ void pl_set_bases(const float* cdf, Assigner<K>* A, uint32_t* Bs, uint32_t kind,
                             const Warp* wp = nullptr) {
  __shared__ int32_t red[32];
  const uint32_t M = A->M, B = A->B;
  const float span = (float)(B - 2u);
  for (uint32_t t = threadIdx.x; t <= M; t += blockDim.x) {
    float f = fminf(fmaxf(cdf[t], 0.0f), 1.0f);
    if (wp && wp->n > 2u) f = warp_fwd(*wp, f);  // focus the buckets on the ks' windows
    Bs[t] = 1u + __float2uint_rn(f * span);
  }
  __syncthreads();
  strict_bases(Bs, M + 1u, B, red);
  if (threadIdx.x == 0) A->kind = kind;
  __syncthreads();
  for (uint32_t t = threadIdx.x; t <= M; t += blockDim.x) {
    A->base[t] = Bs[t];
    if (t < M) {
      const float db = (float)(Bs[t + 1] - Bs[t]);
      const float dx = key_to_float_rn((K)(A->x[t + 1] - A->x[t]));
      A->slope[t] = __fdiv_rn(db, dx);
    }
  }
  __syncthreads();
}

template <typename K>
struct LearnSmem {
  SetupSmem<K> su;
  PLStats st[PL_M];
  PLRed red;
  float cdf[PL_M + 1];
  uint32_t Bs[ASG_MAXM + 1];
  uint32_t q[PL_M + 1];
  float qcdf[PL_M + 1];
  uint32_t seg_start[PL_M + 1];
};

// Knots of the learned models: at most B/4 of them (every segment keeps at
// least a few buckets, and strictly increasing bases fit in [1, B-1]).
__host__ __device__ constexpr uint32_t pl_knots_for(uint32_t B) {
  return (B / 4u) < (uint32_t)PL_M ? (B / 4u) : (uint32_t)PL_M;
}
// The PL model's default: 512 segments (128 sample keys each at S = 65536).
// Measured on 2^28 half-normal keys with 1026 clustered ks: its set-up is
// ~6 us shorter than with 1024, for 4 % more candidates; the MLP keeps the
// B/4 default.
constexpr uint32_t PL_DEFAULT_KNOTS = 512;

// Quantile knots: q_j = round(j * (S - 1) / M), initial CDF j / M.
template <typename K>
__device__ void pl_knots(const K* sorted, uint32_t S, uint32_t B, uint32_t kind, Assigner<K>* A,
                         LearnSmem<K>& sm, uint32_t mreq = 0) {
  const uint32_t Mq = mreq ? min(pl_knots_for(B), mreq)
                           : (kind == GGMS_ASSIGNER_LEARNED_PL ? min(pl_knots_for(B), PL_DEFAULT_KNOTS)
                                                               : pl_knots_for(B));
  for (uint32_t j = threadIdx.x; j <= Mq; j += blockDim.x) {
    sm.q[j] = (uint32_t)(((uint64_t)j * (S - 1u) + Mq / 2) / Mq);
    sm.qcdf[j] = (float)j / (float)Mq;
  }
  __syncthreads();
  asg_build_from_knots<K>(sorted, sm.q, sm.qcdf, Mq, B, kind, A);
  __syncthreads();
}

// Final stage shared by both learned models: compile the PL assigner A into
// the grid G, measure it on the sample and decide learned vs sampled.
// The learned grid is used when its imbalance is within the bound, or when the
// sampled grid G0 (measured the same way on the same sample) is worse still.
// A focused model is measured in CDF space before its warp.
template <typename K>
__device__ void learned_finish(const K* sorted, uint32_t S, uint32_t B, uint32_t kind, float bound,
                               Assigner<K>* A, Grid<K>* G, const Grid<K>* G0, LearnState* L,
                               uint32_t* choice, LearnSmem<K>& sm, const Warp* wp = nullptr) {
  const AsgView<K> av = asg_copy<K>(A, sm.su.asg);
  GGMS_TRACE(14);
  const GridView<K> gv = grid_compile<K>(av, B, kind, G, sm.su.s1, sm.su.s2, sm.su.cs);
  GGMS_TRACE(15);
  const float qv = grid_measure<K>(gv, sorted, S, sm.su.hist256, wp);
  GGMS_TRACE(16);
  if (threadIdx.x == 0) {
    G->quality = qv;
    const uint32_t c = (qv <= bound || qv < G0->quality) ? 1u : 0u;
    *choice = c;
    L->choice = c;
    L->imbalance = qv;
  }
}

// The whole learned-PL setup in one CTA: knots -> statistics -> training ->
// bases -> grid -> occupancy -> choice (grid 1 if within the bound, else the
// sampled grid 0 stays in use).
// Knots of the learned PL model (one CTA): mreq segments requested (0: the
// default, min(PL_DEFAULT_KNOTS, B / 4)).  Launched with two CTAs: CTA 0 places the knots
// while CTA 1 builds the bucket focus from the ks (krank: their ascending ranks
// among n keys; window_z < 0: none) and stores it in L for setup_learned_pl
// (L == null: not stored).
template <typename K>
__global__ __launch_bounds__(SETUP_NT) void setup_pl_knots(const K* __restrict__ sorted, uint32_t S,
                                                          uint32_t B, Assigner<K>* A, uint32_t mreq,
                                                          const uint32_t* __restrict__ krank, uint32_t nk,
                                                          uint64_t n, float window_z, LearnState* L) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem[];
  LearnSmem<K>& sm = *reinterpret_cast<LearnSmem<K>*>(smem);
  __shared__ Warp wsh;
  __shared__ uint32_t wred[33];
  GGMS_TRACE(5);
  if (blockIdx.x == 1) {
    if (!L) return;
    if (window_z >= 0.0f) {
      // the statistics' space is unused in this CTA: it holds the focus bins
      build_warp(krank, nk, n, S, window_z, L0_WIN, reinterpret_cast<uint32_t*>(sm.st), wred, &wsh);
    } else if (threadIdx.x == 0) {
      wsh.n = 2;
      wsh.p[0] = wsh.w[0] = 0.0f;
      wsh.p[1] = wsh.w[1] = 1.0f;
    }
    __syncthreads();
    if (threadIdx.x == 0) L->warp = wsh;
    return;
  }
  pl_knots<K>(sorted, S, B, GGMS_ASSIGNER_LEARNED_PL, A, sm, mreq);
  GGMS_TRACE(6);
}

// Training and compilation of the learned PL model (one CTA), after
// setup_pl_knots and pl_stats_grid.  With window_z >= 0 the bases are focused
// on the ks' windows (build_warp): krank[0..nk) are the ks' ascending ranks
// among n keys.
template <typename K>
__global__ __launch_bounds__(SETUP_NT) void setup_learned_pl(const K* __restrict__ sorted, uint32_t S,
                                                            uint32_t B, uint32_t steps, float lr,
                                                            float bound, Assigner<K>* A, Grid<K>* G,
                                                            const Grid<K>* G0, LearnState* L,
                                                            uint32_t* choice,
                                                            const uint32_t* __restrict__ krank,
                                                            uint32_t nk, uint64_t n, float window_z) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem[];
  LearnSmem<K>& sm = *reinterpret_cast<LearnSmem<K>*>(smem);
  __shared__ Warp wsh;
  const uint32_t M = A->M;  // knots: setup_pl_knots; statistics: pl_stats_grid
  GGMS_TRACE(9);
  pl_stats_load(L, M, sm.st);
  GGMS_TRACE(10);
  __shared__ uint32_t in_alt;
  if (threadIdx.x < PL_NT) {
    // sm.qcdf (the knot placement's scratch) is free here: the second CDF buffer
    const float loss = pl_train_block(sm.st, M, S, steps, lr, sm.red, sm.cdf, sm.qcdf, &in_alt,
                                      &L->loss_init, L->theta, L->grad);
    if (threadIdx.x == 0) {
      L->loss = loss;
      L->M = M;
      L->steps = steps;
    }
  }
  __syncthreads();
  if (in_alt) {
    for (uint32_t j = threadIdx.x; j <= M; j += blockDim.x) sm.cdf[j] = sm.qcdf[j];
    __syncthreads();
  }
  GGMS_TRACE(11);
  if (threadIdx.x == 0) wsh = L->warp;  // built with the knots (setup_pl_knots)
  __syncthreads();
  GGMS_TRACE(12);
  if (threadIdx.x == 0) L->focus_points = wsh.n;
  pl_set_bases<K>(sm.cdf, A, sm.Bs, GGMS_ASSIGNER_LEARNED_PL, &wsh);
  GGMS_TRACE(13);
  learned_finish<K>(sorted, S, B, GGMS_ASSIGNER_LEARNED_PL, bound, A, G, G0, L, choice, sm, &wsh);
}

// Gradient probe (diagnostics): after setup_pl_knots and pl_stats_grid, one
// forward/backward at the given theta -- the kernels training uses.
template <typename K>
__global__ __launch_bounds__(SETUP_NT) void pl_grad_probe(const Assigner<K>* __restrict__ A, uint32_t S,
                                                         const LearnState* L,
                                                         const float* __restrict__ theta_in,
                                                         float* loss_out, float* grad_out) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem[];
  LearnSmem<K>& sm = *reinterpret_cast<LearnSmem<K>*>(smem);
  const uint32_t M = A->M;
  pl_stats_load(L, M, sm.st);
  if (threadIdx.x < PL_NT) {
    float g = 0.0f;
    const float th = threadIdx.x < M ? theta_in[threadIdx.x] : 0.0f;
    const float loss = pl_fb(th, sm.st, M, (double)S, sm.red, &g, nullptr);
    if (threadIdx.x < M) grad_out[threadIdx.x] = g;
    if (threadIdx.x == 0) *loss_out = loss;
  }
}

GGMS_END

#include "ggms_mlp.cuh"

GGMS_BEGIN

template <typename K>
static int learn_and_choose(int kind, const K* sorted, uint32_t S, uint32_t B, int steps_opt,
                            float bound, Assigner<K>* As, Grid<K>* Gs, LearnState* L,
                            uint32_t* choice, const uint32_t* krank, uint32_t nk, uint64_t n,
                            float window_z, cudaStream_t st, long long* launches,
                            cudaEvent_t sampled_done = nullptr, uint32_t pl_knots = 0) {
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(setup_learned_pl<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(LearnSmem<K>)) != cudaSuccess ||
        cudaFuncSetAttribute(setup_pl_knots<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(LearnSmem<K>)) != cudaSuccess)
      return GGMS_E_CUDA;
    attr = true;
  }
  if (kind == GGMS_ASSIGNER_LEARNED_MLP) {
    int rc = mlp_fit_and_compile<K>(sorted, S, B, steps_opt, bound, As, Gs, L, choice, st, launches,
                                    sampled_done, pl_knots);
    if (rc) return rc;
  } else {
    const uint32_t steps = steps_opt > 0 ? (uint32_t)steps_opt : 1u;
    if (launch_pdl(setup_pl_knots<K>, 2, SETUP_NT, sizeof(LearnSmem<K>), st, sorted, S, B, &As[1], pl_knots, krank,
                   nk, n, window_z, L) != cudaSuccess ||
        launch_pdl(pl_stats_grid<K>, (PL_M + 31) / 32, 1024, 0, st, sorted, S, (const Assigner<K>*)&As[1], L) !=
            cudaSuccess)
      return GGMS_E_CUDA;
    // the choice compares with the sampled grid: wait for it (it may be built
    // on another stream, concurrently with the knots and the statistics)
    if (sampled_done && cudaStreamWaitEvent(st, sampled_done, 0) != cudaSuccess) return GGMS_E_CUDA;
    if (launch_pdl(setup_learned_pl<K>, 1, SETUP_NT, sizeof(LearnSmem<K>), st, sorted, S, B, steps, 0.02f, bound,
                   &As[1], &Gs[1], (const Grid<K>*)&Gs[0], L, choice, krank, nk, n, window_z) != cudaSuccess)
      return GGMS_E_CUDA;
    *launches += 3;
  }
  return cudaGetLastError() == cudaSuccess ? GGMS_OK : GGMS_E_CUDA;
}

GGMS_END
