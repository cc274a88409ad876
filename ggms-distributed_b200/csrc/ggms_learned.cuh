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
// PL-CDF model (M <= 256 segments between knots at sample quantiles):
//   delta_j = softplus(theta_j) > 0,  P_j = sum_{t<j} delta_t,  D = sum_t delta_t
//   F(s) = (P_j + u(s) * delta_j) / D   for s in segment j, u = (s - x_j)/(x_{j+1} - x_j)
//   loss = 1/S * sum_i (F(s_i) - y_i)^2,  y_i = (i + 0.5) / S  (sorted sample)
// The loss and its gradient depend on the data only through six per-segment
// sums (n, sum u, sum u^2, sum y, sum y u, sum y^2), gathered once by
// pl_stats; every optimizer step is then O(M) work in one warp (pl_train).
//
// MLP-CDF model (1-32-32-1, monotone): see ggms_mlp.cuh.
#pragma once
#include "ggms_kernels.cuh"

namespace ggms {

constexpr int PL_M = 256;        // segments of the learned PL model
constexpr int MLP_H = 32;        // hidden width of the MLP model
constexpr int MLP_NPARAM = 1153; // 32 + 32 + 32*32 + 32 + 32 + 1

struct PLStats {                 // per segment, in double for a stable sum
  double n, su, su2, sy, syu, sy2;
};

struct LearnState {
  float theta[PL_M];             // PL parameters
  float m1[PL_M], m2[PL_M];      // Adam moments
  float grad[PL_M];              // last gradient w.r.t. theta
  float cdf[PL_M + 1];           // trained CDF at the knots
  PLStats stats[PL_M];
  float loss_init;               // loss before training
  float loss;                    // loss after training
  float imbalance;               // max/mean of the compiled model on the sample
  uint32_t M;                    // segments actually used
  uint32_t steps;
  uint32_t choice;               // 1 learned accepted, 0 fell back to sampled
  uint32_t pad[2];
  // MLP parameters (see ggms_mlp.cuh)
  float mlp_params[MLP_NPARAM + 3];
  float mlp_loss;
};

__device__ __forceinline__ float softplusf(float x) {
  return x > 20.0f ? x : log1pf(expf(x));
}
__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + expf(-x)); }

// Quantile knots: q_j = round(j * (S - 1) / M), initial CDF j / M.
template <typename K>
__global__ void pl_init_knots(const K* __restrict__ sorted, uint32_t S, uint32_t B,
                              Assigner<K>* A) {
  __shared__ uint32_t q[PL_M + 1];
  __shared__ float cdf[PL_M + 1];
  for (uint32_t j = threadIdx.x; j <= (uint32_t)PL_M; j += blockDim.x) {
    q[j] = (uint32_t)(((uint64_t)j * (S - 1u) + PL_M / 2) / PL_M);
    cdf[j] = (float)j / (float)PL_M;
  }
  __syncthreads();
  asg_build_from_knots<K>(sorted, q, cdf, PL_M, B, GGMS_ASSIGNER_LEARNED_PL, A);
}

// Per-segment sufficient statistics of the sorted sample (deterministic: one
// warp per segment, fixed summation order).
template <typename K>
__global__ void pl_stats(const K* __restrict__ sorted, uint32_t S, const Assigner<K>* __restrict__ A,
                         LearnState* L) {
  const uint32_t M = A->M;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (warp >= M) return;
  // samples of segment j: x_j <= s < x_{j+1} (the last segment also takes s == x_M)
  auto lower = [&](K v) {
    uint32_t lo = 0, hi = S;
    while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (sorted[m] < v) lo = m + 1; else hi = m; }
    return lo;
  };
  const K xj = A->x[warp], xn = A->x[warp + 1];
  const uint32_t i0 = lower(xj);
  const uint32_t i1 = (warp + 1 == M) ? S : lower(xn);
  const float width = key_to_float_rn((K)(xn - xj));
  double n = 0, su = 0, su2 = 0, sy = 0, syu = 0, sy2 = 0;
  for (uint32_t i = i0 + lane; i < i1; i += 32) {
    float u = fminf(__fdiv_rn(key_to_float_rn((K)(sorted[i] - xj)), width), 1.0f);
    double y = ((double)i + 0.5) / (double)S;
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
  if (lane == 0) L->stats[warp] = PLStats{n, su, su2, sy, syu, sy2};
}

// Forward + backward of the PL model on the statistics, one warp, M <= 256,
// in double (the loss is a small difference of O(n) sums).  Returns the loss;
// fills g (gradient w.r.t. theta) and, if asked, the CDF at the knots.
// Lane l owns segments [l*PER, l*PER + PER).
__device__ float pl_forward_backward(const float* theta, const PLStats* st, uint32_t M, double S,
                                     float* g, float* cdf_out) {
  constexpr int PER = PL_M / 32;
  const uint32_t lane = threadIdx.x & 31;
  double d[PER], P[PER];
  double local = 0.0;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    uint32_t j = lane * PER + u;
    d[u] = j < M ? (double)softplusf(theta[j]) : 0.0;
    local += d[u];
  }
  double incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double t = __shfl_up_sync(FULL, incl, o);
    if ((int)lane >= o) incl += t;
  }
  const double D = __shfl_sync(FULL, incl, 31);
  double run = incl - local;
#pragma unroll
  for (int u = 0; u < PER; ++u) { P[u] = run; run += d[u]; }
  double R[PER], U[PER];
  double Q = 0.0, loss = 0.0;
  const double invD = 1.0 / D;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    uint32_t j = lane * PER + u;
    R[u] = 0.0; U[u] = 0.0;
    if (j >= M) continue;
    const PLStats s = st[j];
    const double p = P[u] * invD, dd = d[u] * invD;
    // F_i = p + dd * u_i ;  r_i = F_i - y_i
    R[u] = s.n * p + dd * s.su - s.sy;
    U[u] = p * s.su + dd * s.su2 - s.syu;
    const double sF2 = s.n * p * p + 2.0 * p * dd * s.su + dd * dd * s.su2;
    const double sFy = p * s.sy + dd * s.syu;
    Q += sF2 - sFy;
    loss += sF2 - 2.0 * sFy + s.sy2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Q += __shfl_xor_sync(FULL, Q, o);
    loss += __shfl_xor_sync(FULL, loss, o);
  }
  // dF_i/d delta_t = (1{t < j_i} + u_i 1{t = j_i} - F_i) / D
  double rl = 0.0;
#pragma unroll
  for (int u = 0; u < PER; ++u) rl += R[u];
  double rin = rl;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double t = __shfl_up_sync(FULL, rin, o);
    if ((int)lane >= o) rin += t;
  }
  const double rtot = __shfl_sync(FULL, rin, 31);
  double after = rtot - rin;  // sum of R over later lanes
  const double scale = 2.0 / (S * D);
#pragma unroll
  for (int u = PER - 1; u >= 0; --u) {
    uint32_t j = lane * PER + u;
    if (j < M) {
      double gd = scale * (after + U[u] - Q);
      g[j] = (float)(gd * (double)sigmoidf_(theta[j]));
      if (cdf_out) cdf_out[j] = (float)(P[u] * invD);
    }
    after += R[u];
  }
  if (cdf_out && lane == 0) cdf_out[M] = 1.0f;
  return (float)(loss / S);
}

// Adam on theta, one warp.  lr and step count chosen by the host.
__global__ void pl_train(LearnState* L, const uint32_t* __restrict__ Mp, uint32_t S, uint32_t steps,
                         float lr) {
  __shared__ float theta[PL_M], g[PL_M];
  const uint32_t M = *Mp;
  const uint32_t lane = threadIdx.x;
  for (uint32_t j = lane; j < PL_M; j += 32) {
    theta[j] = 0.5413248546f;  // softplus^-1(1): uniform increments = the quantile init
    L->m1[j] = 0.0f;
    L->m2[j] = 0.0f;
  }
  __syncwarp();
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float b1t = 1.0f, b2t = 1.0f;
  float loss0 = pl_forward_backward(theta, L->stats, M, (double)S, g, nullptr);
  __syncwarp();
  float loss = loss0;
  for (uint32_t it = 0; it < steps; ++it) {
    b1t *= b1;
    b2t *= b2;
    for (uint32_t j = lane; j < M; j += 32) {
      float m1 = b1 * L->m1[j] + (1.0f - b1) * g[j];
      float m2 = b2 * L->m2[j] + (1.0f - b2) * g[j] * g[j];
      L->m1[j] = m1;
      L->m2[j] = m2;
      float mh = m1 / (1.0f - b1t), vh = m2 / (1.0f - b2t);
      theta[j] -= lr * mh / (sqrtf(vh) + eps);
    }
    __syncwarp();
    loss = pl_forward_backward(theta, L->stats, M, (double)S, g, nullptr);
    __syncwarp();
  }
  pl_forward_backward(theta, L->stats, M, (double)S, g, L->cdf);
  for (uint32_t j = lane; j < PL_M; j += 32) {
    L->theta[j] = theta[j];
    L->grad[j] = g[j];
  }
  if (lane == 0) {
    L->loss_init = loss0;
    L->loss = loss;
    L->M = M;
    L->steps = steps;
  }
}

// Gradient probe used by the tests: forward/backward at the given theta.
__global__ void pl_grad_probe(LearnState* L, const float* __restrict__ theta_in, uint32_t M,
                              uint32_t S, float* loss_out, float* grad_out) {
  __shared__ float theta[PL_M], g[PL_M];
  for (uint32_t j = threadIdx.x; j < PL_M; j += 32) theta[j] = j < M ? theta_in[j] : 0.0f;
  __syncwarp();
  float loss = pl_forward_backward(theta, L->stats, M, (double)S, g, nullptr);
  __syncwarp();
  for (uint32_t j = threadIdx.x; j < M; j += 32) grad_out[j] = g[j];
  if (threadIdx.x == 0) *loss_out = loss;
}

// Compile trained CDF values at the knots into bases + slopes (same knots, same
// cell table), with strictly increasing bases.
template <typename K>
__global__ void pl_compile(const float* __restrict__ cdf, Assigner<K>* A, uint32_t kind) {
  __shared__ uint32_t Bs[ASG_MAXM + 1];
  const uint32_t M = A->M, B = A->B;
  if (threadIdx.x == 0) {
    const float span = (float)(B - 2u);
    for (uint32_t t = 0; t <= M; ++t) {
      float f = fminf(fmaxf(cdf[t], 0.0f), 1.0f);
      Bs[t] = 1u + __float2uint_rn(f * span);
    }
    Bs[0] = 1u;
    for (uint32_t t = 1; t <= M; ++t) Bs[t] = max(Bs[t], Bs[t - 1] + 1u);
    Bs[M] = max(Bs[M], B - 1u);
    for (int t = (int)M; t >= 0; --t) Bs[t] = min(Bs[t], (B - 1u) - (M - (uint32_t)t));
    if (M == 0) Bs[0] = 1u;
    A->kind = kind;
  }
  __syncthreads();
  for (uint32_t t = threadIdx.x; t <= M; t += blockDim.x) {
    A->base[t] = Bs[t];
    if (t < M) {
      float db = (float)(Bs[t + 1] - Bs[t]);
      float dx = key_to_float_rn((K)(A->x[t + 1] - A->x[t]));
      A->slope[t] = __fdiv_rn(db, dx);
    }
  }
}

template <typename K>
__global__ void asg_measure_kernel(const K* __restrict__ sorted, uint32_t S, Assigner<K>* A) {
  asg_measure<K>(sorted, S, A);
}

// learned accepted if its imbalance is within the bound
template <typename K>
__global__ void asg_choose(Assigner<K>* As, LearnState* L, float bound, uint32_t* choice) {
  const float q = As[1].quality;
  const uint32_t c = (q <= bound) ? 1u : 0u;
  *choice = c;
  L->choice = c;
  L->imbalance = q;
}

}  // namespace ggms

#include "ggms_mlp.cuh"

namespace ggms {

template <typename K>
static int learn_and_choose(int kind, const K* sorted, uint32_t S, uint32_t B, int steps_opt,
                            float bound, Assigner<K>* As, LearnState* L, uint32_t* choice,
                            cudaStream_t st, long long* launches) {
  pl_init_knots<K><<<1, 256, 0, st>>>(sorted, S, B, &As[1]);
  *launches += 1;
  if (kind == GGMS_ASSIGNER_LEARNED_MLP) {
    int rc = mlp_fit_and_compile<K>(sorted, S, steps_opt, As, L, st, launches);
    if (rc) return rc;
  } else {
    const uint32_t steps = steps_opt > 0 ? (uint32_t)steps_opt : 64u;
    pl_stats<K><<<(PL_M * 32 + 255) / 256, 256, 0, st>>>(sorted, S, &As[1], L);
    pl_train<<<1, 32, 0, st>>>(L, &As[1].M, S, steps, 0.05f);
    pl_compile<K><<<1, 256, 0, st>>>(L->cdf, &As[1], GGMS_ASSIGNER_LEARNED_PL);
    *launches += 3;
  }
  asg_measure_kernel<K><<<1, 1024, 0, st>>>(sorted, S, &As[1]);
  asg_choose<K><<<1, 1, 0, st>>>(As, L, bound, choice);
  *launches += 2;
  return cudaGetLastError() == cudaSuccess ? GGMS_OK : GGMS_E_CUDA;
}

}  // namespace ggms
