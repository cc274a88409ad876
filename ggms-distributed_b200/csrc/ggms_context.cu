// ggms_context.cu -- the C ABI of contexts, options, status, profiling and
// the learned-model diagnostics (include/ggms.h, include/ggms_diag.h).  The
// selection entry points are in ggms_f32.cu, ggms_f64.cu, ggms_u32.cu and
// ggms_i32.cu, one translation unit per value type.
#define GGMS_TU tu_ctx
#include "ggms_engine.cuh"
#include "../../include/ggms_diag.h"

GGMS_BEGIN

// ------------------------------------------------------------------ diagnostics
namespace diag {

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
};

static int pl_gradient(const uint32_t* keys, int S, const float* theta, float* loss, float* grad,
                       uint32_t* knots, int* Mout) {
  if (!keys || S < 2 || S > 65536 || !theta || !loss || !grad) return GGMS_E_INVALID_ARG;
  DevBuf dk, da, dt, dout, dl;
  GGMS_CU(cudaMalloc(&dk.p, 4ull * S));
  GGMS_CU(cudaMalloc(&da.p, sizeof(Assigner<uint32_t>)));
  GGMS_CU(cudaMalloc(&dl.p, sizeof(LearnState)));
  GGMS_CU(cudaMalloc(&dt.p, 4ull * PL_M));
  GGMS_CU(cudaMalloc(&dout.p, 4ull * (PL_M + 1)));
  GGMS_CU(cudaMemcpy(dk.p, keys, 4ull * S, cudaMemcpyHostToDevice));
  GGMS_CU(cudaMemcpy(dt.p, theta, 4ull * PL_M, cudaMemcpyHostToDevice));
  auto* A = (Assigner<uint32_t>*)da.p;
  float* dloss = (float*)dout.p;
  float* dgrad = dloss + 1;
  auto* L = (LearnState*)dl.p;
  GGMS_CU(cudaFuncSetAttribute(pl_grad_probe<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(LearnSmem<uint32_t>)));
  GGMS_CU(cudaFuncSetAttribute(setup_pl_knots<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(LearnSmem<uint32_t>)));
  // the same three kernels as training: knots, statistics, forward/backward
  setup_pl_knots<uint32_t><<<2, SETUP_NT, sizeof(LearnSmem<uint32_t>)>>>(
      (const uint32_t*)dk.p, (uint32_t)S, 1u << 14, A, 0u, nullptr, 0u, 0ull, -1.0f, L);
  pl_stats_grid<uint32_t><<<(PL_M + 31) / 32, 1024>>>((const uint32_t*)dk.p, (uint32_t)S, A, L);
  pl_grad_probe<uint32_t><<<1, SETUP_NT, sizeof(LearnSmem<uint32_t>)>>>(A, (uint32_t)S, L,
                                                                         (const float*)dt.p, dloss, dgrad);
  GGMS_CU(cudaDeviceSynchronize());
  Assigner<uint32_t> h;
  GGMS_CU(cudaMemcpy(&h, A, sizeof(h), cudaMemcpyDeviceToHost));
  GGMS_CU(cudaMemcpy(loss, dloss, 4, cudaMemcpyDeviceToHost));
  GGMS_CU(cudaMemcpy(grad, dgrad, 4ull * h.M, cudaMemcpyDeviceToHost));
  if (knots) memcpy(knots, h.x, 4ull * (h.M + 1));
  if (Mout) *Mout = (int)h.M;
  return GGMS_OK;
}

static int mlp_gradient(const float* x, const float* t, const float* params, float* loss, float* grad) {
  if (!x || !t || !params || !loss || !grad) return GGMS_E_INVALID_ARG;
  DevBuf dx, dt, dp, dprobe;
  GGMS_CU(cudaMalloc(&dx.p, 4ull * MLP_Q));
  GGMS_CU(cudaMalloc(&dt.p, 4ull * MLP_Q));
  GGMS_CU(cudaMalloc(&dp.p, 4ull * MLP_NP));
  GGMS_CU(cudaMalloc(&dprobe.p, 4ull * (MLP_NP + 1)));
  GGMS_CU(cudaMemcpy(dx.p, x, 4ull * MLP_Q, cudaMemcpyHostToDevice));
  GGMS_CU(cudaMemcpy(dt.p, t, 4ull * MLP_Q, cudaMemcpyHostToDevice));
  GGMS_CU(cudaMemcpy(dp.p, params, 4ull * MLP_NP, cudaMemcpyHostToDevice));
  GGMS_CU(cudaFuncSetAttribute(mlp_train<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(MlpSmem)));
  mlp_train<uint32_t><<<MLP_CTAS, MLP_NT, sizeof(MlpSmem)>>>(
      nullptr, 0u, nullptr, nullptr, (float*)dp.p, 0u, 0.0f, (const float*)dx.p, (const float*)dt.p,
      (float*)dprobe.p);
  GGMS_CU(cudaDeviceSynchronize());
  float* hp = (float*)malloc(4ull * (MLP_NP + 1));
  if (!hp) return GGMS_E_OOM;
  cudaError_t e = cudaMemcpy(hp, dprobe.p, 4ull * (MLP_NP + 1), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) {
    memcpy(grad, hp, 4ull * MLP_NP);
    *loss = hp[MLP_NP];
  }
  free(hp);
  return cuda_status(e);
}

static int fit(const uint32_t* keys, int S, int kind, int steps, float* l0, float* l1, float* imb_m,
               float* imb_s) {
  if (!keys || S < 1024 || (kind != GGMS_ASSIGNER_LEARNED_PL && kind != GGMS_ASSIGNER_LEARNED_MLP))
    return GGMS_E_INVALID_ARG;
  DevBuf dk, da, dg, dl, dc;
  GGMS_CU(cudaMalloc(&dk.p, 4ull * S));
  GGMS_CU(cudaMalloc(&da.p, 2 * sizeof(Assigner<uint32_t>)));
  GGMS_CU(cudaMalloc(&dg.p, 2 * sizeof(Grid<uint32_t>)));
  GGMS_CU(cudaMalloc(&dl.p, sizeof(LearnState)));
  GGMS_CU(cudaMalloc(&dc.p, 4));
  GGMS_CU(cudaMemcpy(dk.p, keys, 4ull * S, cudaMemcpyHostToDevice));
  auto* As = (Assigner<uint32_t>*)da.p;
  auto* Gs = (Grid<uint32_t>*)dg.p;
  auto* L = (LearnState*)dl.p;
  const uint32_t* k = (const uint32_t*)dk.p;
  const uint32_t B = 1u << 14;
  int rc = setup_attrs<uint32_t>();
  if (rc) return rc;
  setup_sampled<uint32_t><<<1, SETUP_NT, sizeof(SetupSmem<uint32_t>)>>>(k, (uint32_t)S, B, &As[0], &Gs[0]);
  long long launches = 0;
  rc = learn_and_choose<uint32_t>(kind, k, (uint32_t)S, B, steps, 1e30f, As, Gs, L, (uint32_t*)dc.p,
                                  nullptr, 0u, 0ull, -1.0f, 0, &launches);
  if (rc) return rc;
  GGMS_CU(cudaDeviceSynchronize());
  LearnState hl;
  Grid<uint32_t> a0, a1;
  GGMS_CU(cudaMemcpy(&hl, L, sizeof(hl), cudaMemcpyDeviceToHost));
  GGMS_CU(cudaMemcpy(&a0, &Gs[0], sizeof(a0), cudaMemcpyDeviceToHost));
  GGMS_CU(cudaMemcpy(&a1, &Gs[1], sizeof(a1), cudaMemcpyDeviceToHost));
  if (l0) *l0 = (kind == GGMS_ASSIGNER_LEARNED_PL) ? hl.loss_init : -1.0f;
  if (l1) *l1 = (kind == GGMS_ASSIGNER_LEARNED_PL) ? hl.loss : hl.mlp_loss;
  if (imb_m) *imb_m = a1.quality;
  if (imb_s) *imb_s = a0.quality;
  return GGMS_OK;
}

}  // namespace diag

GGMS_END

using namespace ggms;

extern "C" {

void ggms_default_opts(ggms_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->struct_size = (int32_t)sizeof(ggms_opts);
  o->assigner = GGMS_ASSIGNER_AUTO;
  o->seed = 0x5EEDull;
  o->imbalance_bound = 3.0f;
}

const char* ggms_status_string(int s) {
  switch (s) {
    case GGMS_OK: return "ok";
    case GGMS_E_INVALID_ARG: return "invalid argument";
    case GGMS_E_OOM: return "out of memory";
    case GGMS_E_NOT_CONVERGED: return "not converged";
    case GGMS_E_CUDA: return "CUDA error";
    case GGMS_E_UNSUPPORTED: return "unsupported";
    case GGMS_E_INTERNAL: return "internal error";
    default: return "unknown status";
  }
}

int ggms_version(void) { return 200; }

int ggms_create(ggms_context** ctx, int device) {
  if (!ctx) return GGMS_E_INVALID_ARG;
  Context* c = nullptr;
  int rc = create_context(&c, device);
  if (rc) return rc;
  *ctx = (ggms_context*)c;
  return GGMS_OK;
}

int ggms_destroy(ggms_context* ctx) {
  destroy_context((Context*)ctx);
  return GGMS_OK;
}

int ggms_get_default_context(ggms_context** ctx) {
  if (!ctx) return GGMS_E_INVALID_ARG;
  Context* c = nullptr;
  int rc = default_context(&c);
  if (rc) return rc;
  *ctx = (ggms_context*)c;
  return GGMS_OK;
}

int ggms_context_profile(ggms_context* ctx, int enable) {
  Context* c = (Context*)ctx;
  if (!c) return GGMS_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  c->profile = enable != 0;
  return GGMS_OK;
}

int ggms_context_pass_times(ggms_context* ctx, float* p1, float* p2, float* call, int max) {
  Context* c = (Context*)ctx;
  if (!c || max < 0) return -GGMS_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  int got = 0;
  while (c->ring_count > 0 && got < max) {
    cudaEvent_t* e = c->ev[c->ring_head];
    if (cudaEventSynchronize(e[5]) != cudaSuccess) return -GGMS_E_CUDA;
    float a = 0, b = 0, t = 0;
    cudaEventElapsedTime(&a, e[1], e[2]);
    cudaEventElapsedTime(&b, e[3], e[4]);
    cudaEventElapsedTime(&t, e[0], e[5]);
    if (p1) p1[got] = a;
    if (p2) p2[got] = b;
    if (call) call[got] = t;
    ++got;
    c->ring_head = (c->ring_head + 1) % Context::RING;
    c->ring_count--;
  }
  return got;
}

int ggms_context_phase_times(ggms_context* ctx, float* ms, int max) {
  Context* c = (Context*)ctx;
  if (!c || max < 0 || (!ms && max > 0)) return -GGMS_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  // phase j runs from boundary event a[j] to b[j] (indices into the call's events)
  static const int a[GGMS_PHASES] = {0, 6, 7, 1, 2, 3, 4, 8};
  static const int b[GGMS_PHASES] = {6, 7, 1, 2, 3, 4, 8, 5};
  int got = 0;
  while (c->ring_count > 0 && got < max) {
    cudaEvent_t* e = c->ev[c->ring_head];
    if (cudaEventSynchronize(e[5]) != cudaSuccess) return -GGMS_E_CUDA;
    for (int j = 0; j < GGMS_PHASES; ++j) {
      float t = 0.0f;
      cudaEventElapsedTime(&t, e[a[j]], e[b[j]]);
      ms[(size_t)got * GGMS_PHASES + j] = t;
    }
    ++got;
    c->ring_head = (c->ring_head + 1) % Context::RING;
    c->ring_count--;
  }
  return got;
}

int ggms_context_status(ggms_context* ctx, void* stream, int* status) {
  Context* c = (Context*)ctx;
  if (!c || !status) return GGMS_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  *status = GGMS_OK;
  if (!c->has_done || !c->arena) return GGMS_OK;  // no call enqueued yet
  GGMS_CU(cudaSetDevice(c->device));
  if (!c->query) GGMS_CU(cudaStreamCreateWithFlags(&c->query, cudaStreamNonBlocking));
  GGMS_CU(cudaStreamWaitEvent(c->query, c->done, 0));
  if (stream) {
    cudaEvent_t e;
    GGMS_CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaError_t r = cudaEventRecord(e, (cudaStream_t)stream);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(c->query, e, 0);
    cudaEventDestroy(e);
    GGMS_CU(r);
  }
  uint32_t word = 0;
  GGMS_CU(cudaMemcpyAsync(&word, &((const Counters*)c->arena)->status, sizeof(word),
                          cudaMemcpyDeviceToHost, c->query));
  GGMS_CU(cudaStreamSynchronize(c->query));
  *status = (int)word;
  return GGMS_OK;
}

int64_t ggms_context_launches(ggms_context* ctx) {
  Context* c = (Context*)ctx;
  if (!c) return -1;
  return (int64_t)c->launches;
}

int64_t ggms_context_graph_launches(ggms_context* ctx) {
  Context* c = (Context*)ctx;
  if (!c) return -1;
  std::lock_guard<std::mutex> lk(c->mu);
  return c->graph_launches;
}

int ggms_diag_pl_gradient(const uint32_t* keys, int S, const float* theta, float* loss, float* grad,
                          uint32_t* knots, int* M) {
  return diag::pl_gradient(keys, S, theta, loss, grad, knots, M);
}

int ggms_diag_mlp_gradient(const float* x, const float* t, const float* params, float* loss,
                           float* grad) {
  return diag::mlp_gradient(x, t, params, loss, grad);
}

int ggms_diag_fit(const uint32_t* keys, int S, int kind, int steps, float* l0, float* l1,
                  float* imb_m, float* imb_s) {
  return diag::fit(keys, S, kind, steps, l0, l1, imb_m, imb_s);
}

}  // extern "C"

