// ggms_mlp.cuh -- monotone 1-32-32-1 MLP CDF model, trained on the GPU.
//
//   x = F0(key)                      the sampled pivots' piecewise-linear CDF
//                                    (the reference's bucket map), in [0, 1]
//   h1 = tanh(w1 * x + c1)           w1 = softplus(V1) > 0     (32)
//   h2 = tanh(W2 h1 + c2)            W2 = softplus(V2) > 0     (32 x 32)
//   y  = sigmoid(w3 . h2 + c3)       w3 = softplus(V3) > 0
// Positive weights and increasing activations make y non-decreasing in x, and
// F0 is non-decreasing, so y(F0(key)) is monotone in the key and so is the
// compiled assigner.  The network thus learns a monotone correction of the
// sampled model: where the data's density changes inside a pivot interval
// (mixtures, heavy tails) F0 is off and the network bends it back.  Loss:
// mean (z_i - logit t_i)^2 over Q = 1024 training points at the quantiles of
// the self-drawn sample (t_i = (rank + 1/2) / S), i.e. the error of the
// sigmoid's argument.  In logit units the tails weigh as much as the middle:
// a CDF-space error would let the network squeeze the top and bottom percent
// of the keys into a few buckets where the sigmoid saturates (on a lognormal
// sample that made one of 256 bucket groups hold 8x its share).
//
// Training runs in ONE launch of one thread-block cluster (8 CTAs x 128
// threads, one training point per thread): every step each CTA computes its
// partial gradient (per-sample forward/backward, then the weight-gradient
// contractions from shared memory), CTA 0 sums the eight partials through
// distributed shared memory, applies Adam and the other CTAs read the new
// parameters back the same way.  The trained model is evaluated at the knots
// of the PL assigner format and compiled into it (pl_compile).
#pragma once
#include <cooperative_groups.h>


GGMS_BEGIN

namespace cg = cooperative_groups;

constexpr int MLP_CTAS = 8;
constexpr int MLP_NT = 128;
constexpr int MLP_Q = MLP_CTAS * MLP_NT;                 // training points per step
constexpr int MLP_NP = MLP_NPARAM;  // 1153 parameters
static_assert(MLP_NP == MLP_H + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1, "parameter count");
// parameter offsets in the flat vector
constexpr int P_V1 = 0, P_C1 = 32, P_V2 = 64, P_C2 = 64 + 1024, P_V3 = P_C2 + 32, P_C3 = P_V3 + 32;

struct MlpSmem {
  float P[MLP_NP];          // raw parameters (V1, c1, V2, c2, V3, c3)
  float Pbest[MLP_NP];      // best parameters seen (CTA 0)
  float G[MLP_NP + 1];      // this CTA's partial gradient, then its squared-error sum
  float best, cur_loss;
  float m1[MLP_NP], m2[MLP_NP];  // Adam moments (CTA 0)
  float w1[32], W2[1024], w3[32];  // softplus'd weights
  float x[MLP_NT], t[MLP_NT], dz[MLP_NT], err[MLP_NT];
  float h1[MLP_NT][33], h2[MLP_NT][33], da1[MLP_NT][33], da2[MLP_NT][33];
};

__device__ __forceinline__ float tanh_(float v) { return tanhf(v); }

// Forward + backward of this CTA's MLP_NT points; fills S.G with the partial
// gradient (w.r.t. the raw parameters) and S.err with the squared errors.
__device__ void mlp_cta_grad(MlpSmem& S, float inv_q) {
  const int tid = threadIdx.x;
  for (int i = tid; i < 1024; i += MLP_NT) S.W2[i] = softplusf(S.P[P_V2 + i]);
  if (tid < 32) {
    S.w1[tid] = softplusf(S.P[P_V1 + tid]);
    S.w3[tid] = softplusf(S.P[P_V3 + tid]);
  }
  __syncthreads();
  // per-sample forward and backward to the hidden layers
  {
    const float x = S.x[tid];
    float h1[32], h2[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) h1[j] = tanh_(fmaf(S.w1[j], x, S.P[P_C1 + j]));
    float z = S.P[P_C3];
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      float a = S.P[P_C2 + k];
#pragma unroll
      for (int j = 0; j < 32; ++j) a = fmaf(S.W2[k * 32 + j], h1[j], a);
      h2[k] = tanh_(a);
      z = fmaf(S.w3[k], h2[k], z);
    }
    const float e = z - S.t[tid];  // S.t holds logit targets
    S.err[tid] = e * e;
    const float dz = 2.0f * e * inv_q;
    S.dz[tid] = dz;
    float dh1[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) dh1[j] = 0.0f;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const float da2 = dz * S.w3[k] * (1.0f - h2[k] * h2[k]);
      S.da2[tid][k] = da2;
      S.h2[tid][k] = h2[k];
#pragma unroll
      for (int j = 0; j < 32; ++j) dh1[j] = fmaf(S.W2[k * 32 + j], da2, dh1[j]);
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      S.h1[tid][j] = h1[j];
      S.da1[tid][j] = dh1[j] * (1.0f - h1[j] * h1[j]);
    }
  }
  __syncthreads();
  // weight gradients: contractions over the CTA's samples (fixed order)
  for (int p = tid; p < 1024; p += MLP_NT) {
    const int k = p >> 5, j = p & 31;
    float acc = 0.0f;
    for (int i = 0; i < MLP_NT; ++i) acc = fmaf(S.da2[i][k], S.h1[i][j], acc);
    S.G[P_V2 + p] = acc * sigmoidf_(S.P[P_V2 + p]);  // d softplus(v) / dv = sigmoid(v)
  }
  if (tid < 32) {
    float gw1 = 0, gc1 = 0, gc2 = 0, gw3 = 0;
    for (int i = 0; i < MLP_NT; ++i) {
      gw1 = fmaf(S.da1[i][tid], S.x[i], gw1);
      gc1 += S.da1[i][tid];
      gc2 += S.da2[i][tid];
      gw3 = fmaf(S.dz[i], S.h2[i][tid], gw3);
    }
    S.G[P_V1 + tid] = gw1 * sigmoidf_(S.P[P_V1 + tid]);
    S.G[P_C1 + tid] = gc1;
    S.G[P_C2 + tid] = gc2;
    S.G[P_V3 + tid] = gw3 * sigmoidf_(S.P[P_V3 + tid]);
  } else if (tid == 32) {
    float gc3 = 0;
    for (int i = 0; i < MLP_NT; ++i) gc3 += S.dz[i];
    S.G[P_C3] = gc3;
  } else if (tid == 64) {
    float e = 0;
    for (int i = 0; i < MLP_NT; ++i) e += S.err[i];
    S.G[MLP_NP] = e;
  }
  __syncthreads();
}

// The network's input: the sampled model A0's CDF at `key`, the position of the
// key on A0's piecewise-linear bucket map divided by the bucket count
// (continuous, not rounded to a bucket), clamped to [0, 1].
template <typename K>
__device__ __forceinline__ float mlp_input(const Assigner<K>* __restrict__ A0, K key) {
  const uint32_t M = A0->M;
  const K x0 = A0->x[0];
  if (M == 0u || key <= x0) return 0.0f;
  if (key >= A0->x[M]) return 1.0f;
  uint32_t j = A0->idx[(uint32_t)((K)(key - x0) >> A0->csh)];
  while (j + 1u < M && key >= A0->x[j + 1u]) ++j;
  const float b = (float)A0->base[j] + __fmul_rn(key_to_float_rn((K)(key - A0->x[j])), A0->slope[j]);
  return fminf(fmaxf(__fdiv_rn(b, (float)A0->B), 0.0f), 1.0f);
}

__device__ __forceinline__ float logitf_(float t) { return logf(t) - log1pf(-t); }

// Training points: Q sample quantiles, x = F0 of the key, target
// logit((rank + 0.5) / S); explicit points carry CDF targets in (0, 1).
template <typename K>
__device__ void mlp_load_points(MlpSmem& S, const K* sorted, uint32_t S_n, const Assigner<K>* A0,
                                const float* px, const float* pt) {
  const int tid = threadIdx.x;
  const uint32_t gi = blockIdx.x * MLP_NT + tid;
  if (px) {  // explicit points (gradient probe)
    S.x[tid] = px[gi];
    S.t[tid] = logitf_(pt[gi]);
    return;
  }
  const uint32_t si = (uint32_t)(((uint64_t)(2 * gi + 1) * S_n) / (2 * MLP_Q));
  S.x[tid] = mlp_input<K>(A0, sorted[si]);
  S.t[tid] = logitf_(((float)si + 0.5f) / (float)S_n);
}

// The cluster training kernel.  steps == 0 with probe != null: one forward /
// backward at L's parameters, the summed gradient and loss are written to
// probe[0..MLP_NP) and probe[MLP_NP] (used by the gradient check).
template <typename K>
__global__ void __cluster_dims__(MLP_CTAS, 1, 1) __launch_bounds__(MLP_NT)
mlp_train(const K* __restrict__ sorted, uint32_t S_n, const Assigner<K>* __restrict__ A0,
          LearnState* L, float* Pglob, uint32_t steps, float lr, const float* px, const float* pt,
          float* probe) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem_raw[];
  MlpSmem& S = *reinterpret_cast<MlpSmem*>(smem_raw);
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  const int tid = threadIdx.x;
  for (int p = tid; p < MLP_NP; p += MLP_NT) {
    S.P[p] = Pglob[p];
    S.m1[p] = 0.0f;
    S.m2[p] = 0.0f;
  }
  mlp_load_points<K>(S, sorted, S_n, A0, px, pt);
  __syncthreads();
  MlpSmem* S0 = cluster.map_shared_rank(&S, 0);
  const float inv_q = 1.0f / (float)MLP_Q;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float b1t = 1.0f, b2t = 1.0f;
  const uint32_t iters = steps ? steps : 1u;
  if (tid == 0) S.best = 3.0e38f;
  for (uint32_t it = 0; it < iters; ++it) {
    mlp_cta_grad(S, inv_q);
    cluster.sync();  // all partial gradients are in place
    if (rank == 0) {
      if (tid == 0) {
        float e = 0.0f;
        for (unsigned r = 0; r < MLP_CTAS; ++r) e += cluster.map_shared_rank(&S, r)->G[MLP_NP];
        S.cur_loss = e * inv_q;
      }
      __syncthreads();
      const bool better = S.cur_loss < S.best;  // loss at the parameters before this step
      if (better)
        for (int p = tid; p < MLP_NP; p += MLP_NT) S.Pbest[p] = S.P[p];
      b1t *= b1;
      b2t *= b2;
      for (int p = tid; p < MLP_NP; p += MLP_NT) {
        float g = 0.0f;
        for (unsigned r = 0; r < MLP_CTAS; ++r) g += cluster.map_shared_rank(&S, r)->G[p];
        if (steps == 0) {
          if (probe) probe[p] = g;
          continue;
        }
        const float m1 = b1 * S.m1[p] + (1.0f - b1) * g;
        const float m2 = b2 * S.m2[p] + (1.0f - b2) * g * g;
        S.m1[p] = m1;
        S.m2[p] = m2;
        S.P[p] -= lr * (m1 / (1.0f - b1t)) / (sqrtf(m2 / (1.0f - b2t)) + eps);
      }
      __syncthreads();
      if (tid == 0 && better) S.best = S.cur_loss;
    }
    cluster.sync();  // CTA 0 has the new parameters
    if (rank != 0)
      for (int p = tid; p < MLP_NP; p += MLP_NT) S.P[p] = S0->P[p];
    __syncthreads();
  }
  // loss at the final parameters; keep them only if they beat the best seen
  mlp_cta_grad(S, inv_q);
  cluster.sync();
  if (rank == 0) {
    if (tid == 0) {
      float e = 0.0f;
      for (unsigned r = 0; r < MLP_CTAS; ++r) e += cluster.map_shared_rank(&S, r)->G[MLP_NP];
      S.cur_loss = e * inv_q;
      if (probe && steps == 0) probe[MLP_NP] = S.cur_loss;
    }
    __syncthreads();
    const bool use_best = steps > 0 && S.best < S.cur_loss;
    for (int p = tid; p < MLP_NP; p += MLP_NT) Pglob[p] = use_best ? S.Pbest[p] : S.P[p];
    if (tid == 0 && L) L->mlp_loss = use_best ? S.best : S.cur_loss;
  }
  cluster.sync();  // keep every CTA's shared memory alive until CTA 0 has read it
}

// Initial parameters.  Layer 1: unit j is a step at the sample quantile
// q_j = (2j+1)/64 whose width is the local quantile spacing (steep where the
// data is dense), so mean_j (h1_j + 1)/2 already approximates the CDF.  Layer 2:
// unit k steps where that approximation crosses (k + 0.5)/32.  Layer 3: the
// mean of the layer-2 steps through the near-linear part of the sigmoid.
template <typename K>
__device__ void mlp_init(const K* __restrict__ sorted, uint32_t S_n, const Assigner<K>* __restrict__ A0,
                         float* P) {
  const int tid = threadIdx.x;
  auto qx = [&](int j) -> float {  // the input at quantile (2j+1)/64; -1 -> 0, 32 -> 1
    if (j < 0) return 0.0f;
    if (j > 31) return 1.0f;
    const uint32_t si = (uint32_t)(((uint64_t)(2 * j + 1) * S_n) / 64u);
    return mlp_input<K>(A0, sorted[si]);
  };
  for (int p = tid; p < MLP_NP; p += blockDim.x) {
    float v = 0.0f;
    if (p < P_C1) {                       // V1: w1 = 2 / local spacing
      const int j = p - P_V1;
      const float w1 = fminf(2.0f / fmaxf(qx(j + 1) - qx(j - 1), 1e-7f), 1e6f);
      v = w1 + log1pf(-expf(-w1));        // softplus^-1(w1)
    } else if (p < P_V2) {                // c1 = -w1 q_j
      const int j = p - P_C1;
      const float w1 = fminf(2.0f / fmaxf(qx(j + 1) - qx(j - 1), 1e-7f), 1e6f);
      v = -w1 * qx(j);
    } else if (p < P_C2) {                // V2: W2 = 1/32
      v = logf(expm1f(1.0f / 32.0f));
    } else if (p < P_V3) {                // c2: steps at (k + 0.5) / 32
      const int k = p - P_C2;
      v = (1.0f / 32.0f) * (32.0f - 64.0f * ((float)k + 0.5f) / 32.0f);
    } else if (p < P_C3) {                // V3: w3 = 1/16
      v = logf(expm1f(1.0f / 16.0f));
    } else {
      v = 0.0f;                           // c3
    }
    P[p] = v;
  }
}

// Evaluate the trained MLP at the knots of A (input F0 of each knot) and write
// the normalized CDF.
template <typename K>
__device__ void mlp_eval_knots(const float* __restrict__ P, const Assigner<K>* __restrict__ A,
                               const Assigner<K>* __restrict__ A0, float* y, float* cdf) {
  const uint32_t M = A->M;
  for (uint32_t j = threadIdx.x; j <= M; j += blockDim.x) {
    const float x = mlp_input<K>(A0, A->x[j]);
    float h1[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) h1[i] = tanhf(fmaf(softplusf(P[P_V1 + i]), x, P[P_C1 + i]));
    float z = P[P_C3];
    for (int k = 0; k < 32; ++k) {
      float a = P[P_C2 + k];
#pragma unroll
      for (int i = 0; i < 32; ++i) a = fmaf(softplusf(P[P_V2 + k * 32 + i]), h1[i], a);
      z = fmaf(softplusf(P[P_V3 + k]), tanhf(a), z);
    }
    y[j] = sigmoidf_(z);
  }
  __syncthreads();
  const float lo = y[0], hi = y[M];
  for (uint32_t j = threadIdx.x; j <= M; j += blockDim.x)
    cdf[j] = (hi > lo) ? fmaxf((y[j] - lo) / (hi - lo), 0.0f) : (float)j / (float)(M ? M : 1);
  __syncthreads();
}

template <typename K>
__global__ __launch_bounds__(SETUP_NT) void setup_mlp_begin(const K* __restrict__ sorted, uint32_t S,
                                                           uint32_t B, Assigner<K>* A, const Assigner<K>* A0,
                                                           float* P, uint32_t mreq) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem[];
  LearnSmem<K>& sm = *reinterpret_cast<LearnSmem<K>*>(smem);
  pl_knots<K>(sorted, S, B, GGMS_ASSIGNER_LEARNED_MLP, A, sm, mreq);
  mlp_init<K>(sorted, S, A0, P);
}

template <typename K>
__global__ __launch_bounds__(SETUP_NT) void setup_mlp_finish(const K* __restrict__ sorted, uint32_t S,
                                                            uint32_t B, float bound, const float* P,
                                                            Assigner<K>* A, Grid<K>* G, LearnState* L,
                                                            uint32_t* choice) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem[];
  LearnSmem<K>& sm = *reinterpret_cast<LearnSmem<K>*>(smem);
  mlp_eval_knots<K>(P, A, A - 1, (float*)sm.Bs, sm.cdf);  // A - 1: the sampled assigner of the pair
  for (uint32_t j = threadIdx.x; j <= A->M; j += blockDim.x) L->cdf[j] = sm.cdf[j];
  if (threadIdx.x == 0) L->M = A->M;  // segments of the compiled piecewise-linear form
  pl_set_bases<K>(sm.cdf, A, sm.Bs, GGMS_ASSIGNER_LEARNED_MLP);
  // G is the learned slot of the grid pair: G - 1 is the sampled grid
  learned_finish<K>(sorted, S, B, GGMS_ASSIGNER_LEARNED_MLP, bound, A, G, G - 1, L, choice, sm);
}

template <typename K>
static int mlp_fit_and_compile(const K* sorted, uint32_t S, uint32_t B, int steps_opt, float bound,
                               Assigner<K>* As, Grid<K>* Gs, LearnState* L, uint32_t* choice,
                               cudaStream_t st, long long* launches, cudaEvent_t sampled_done,
                               uint32_t pl_knots) {
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(mlp_train<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(MlpSmem)) != cudaSuccess ||
        cudaFuncSetAttribute(setup_mlp_begin<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(LearnSmem<K>)) != cudaSuccess ||
        cudaFuncSetAttribute(setup_mlp_finish<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(LearnSmem<K>)) != cudaSuccess)
      return GGMS_E_CUDA;
    attr_set = true;
  }
  const uint32_t steps = steps_opt > 0 ? (uint32_t)steps_opt : 150u;
  float* P = L->mlp_params;
  // the network's input is the sampled model: wait for it (it may be built on
  // another stream)
  if (sampled_done && cudaStreamWaitEvent(st, sampled_done, 0) != cudaSuccess) return GGMS_E_CUDA;
  setup_mlp_begin<K><<<1, SETUP_NT, sizeof(LearnSmem<K>), st>>>(sorted, S, B, &As[1], &As[0], P, pl_knots);
  mlp_train<K><<<MLP_CTAS, MLP_NT, sizeof(MlpSmem), st>>>(sorted, S, &As[0], L, P, steps, 0.05f,
                                                          nullptr, nullptr, nullptr);
  setup_mlp_finish<K><<<1, SETUP_NT, sizeof(LearnSmem<K>), st>>>(sorted, S, B, bound, P, &As[1],
                                                                  &Gs[1], L, choice);
  *launches += 3;
  return cudaGetLastError() == cudaSuccess ? GGMS_OK : GGMS_E_CUDA;
}

GGMS_END
