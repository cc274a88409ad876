// ggms_host.cuh -- host-side state shared by every translation unit of the
// library: the context (workspace arena, pinned staging, events, captured CUDA
// graphs, autotuner picks), call plans, option parsing and graph replay.
// Nothing here launches a kernel; the kernels and the code that launches them
// live in ggms_engine.cuh, compiled once per value type (ggms_f32.cu, ...).
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

#include "ggms_internal.cuh"
#include "../../include/ggms.h"

namespace ggms {

// ------------------------------------------------------------------ context
struct Context {
  int device = 0;
  int sms = 148;
  uint8_t* arena = nullptr;
  size_t arena_bytes = 0;
  uint8_t* pinned = nullptr;
  size_t pinned_bytes = 0;
  std::mutex mu;
  long long launches = 0;          // kernels launched by this context
  long long graph_launches = 0;    // calls replayed from a captured CUDA graph
  // profiling: events at the phase boundaries of a call (ring of calls):
  // 0 start, 1 PASS 1 start, 2 PASS 1 end, 3 PASS 2 start, 4 PASS 2 end, 5 end,
  // 6 sample sorted, 7 assigner built, 8 finishing done
  static constexpr int RING = 256;
  static constexpr int NEV = 9;
  bool profile = false;
  cudaEvent_t ev[RING][NEV] = {};
  // the last call's completion (ggms_context_status waits for it)
  cudaEvent_t done = nullptr;
  bool has_done = false;
  cudaStream_t query = nullptr;
  int ring_head = 0, ring_count = 0;
  // captured CUDA graphs of repeated calls (same arguments, same workspace)
  struct Graph {
    uint64_t key[16];
    cudaGraphExec_t exec = nullptr;  // null: seen once, not captured yet
    long long launches = 0;
    uint64_t used = 0;
  };
  static constexpr size_t GRAPHS = 8;
  std::vector<Graph> graphs;
  uint64_t clock = 0;
  cudaStream_t capture = nullptr;  // private stream the graphs are captured on
  cudaEvent_t pin_busy = nullptr;  // recorded after the last call's uploads from the pinned buffer
  static constexpr int MAX_NEST = 8;
  cudaStream_t bodies[MAX_NEST] = {};  // private streams the nested level bodies are captured on
  cudaStream_t side = nullptr;     // the sampled assigner's build next to the learned one; the warp finisher
  cudaEvent_t fork = nullptr, join = nullptr, fork2 = nullptr, join2 = nullptr;
  // autotuner: launch shapes and bucket counts picked per shape class
  struct Tuned {
    uint64_t key[4];
    int B, nt, unroll, lv_mult;
  };
  std::vector<Tuned> tuned;
};

static int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return GGMS_OK;
  if (e == cudaErrorMemoryAllocation) return GGMS_E_OOM;
  return GGMS_E_CUDA;
}

#define GGMS_CU(x)                                  \
  do {                                              \
    cudaError_t e_ = (x);                           \
    if (e_ != cudaSuccess) return cuda_status(e_);  \
  } while (0)

static int ensure_arena(Context* c, size_t bytes) {
  if (c->arena_bytes >= bytes) return GGMS_OK;
  if (c->arena) {
    GGMS_CU(cudaDeviceSynchronize());
    cudaFree(c->arena);
    c->arena = nullptr;
    c->arena_bytes = 0;
  }
  size_t want = bytes + bytes / 8;
  GGMS_CU(cudaMalloc(&c->arena, want));
  c->arena_bytes = want;
  return GGMS_OK;
}

static int ensure_pinned(Context* c, size_t bytes) {
  if (c->pinned_bytes >= bytes) return GGMS_OK;
  if (c->pinned) {
    GGMS_CU(cudaDeviceSynchronize());
    cudaFreeHost(c->pinned);
    c->pinned = nullptr;
    c->pinned_bytes = 0;
  }
  size_t want = std::max<size_t>(bytes, 1 << 16);
  GGMS_CU(cudaMallocHost(&c->pinned, want));
  c->pinned_bytes = want;
  return GGMS_OK;
}

static int create_context(Context** out, int device) {
  Context* c = new (std::nothrow) Context();
  if (!c) return GGMS_E_OOM;
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    delete c;
    return cuda_status(e);
  }
  *out = c;
  return GGMS_OK;
}

static void destroy_context(Context* c) {
  if (!c) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  if (c->arena) cudaFree(c->arena);
  if (c->pinned) cudaFreeHost(c->pinned);
  for (int i = 0; i < Context::RING; ++i)
    for (int j = 0; j < Context::NEV; ++j)
      if (c->ev[i][j]) cudaEventDestroy(c->ev[i][j]);
  if (c->done) cudaEventDestroy(c->done);
  if (c->query) cudaStreamDestroy(c->query);
  for (auto& g : c->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (c->capture) cudaStreamDestroy(c->capture);
  if (c->pin_busy) cudaEventDestroy(c->pin_busy);
  for (auto& b : c->bodies)
    if (b) cudaStreamDestroy(b);
  if (c->side) cudaStreamDestroy(c->side);
  for (cudaEvent_t e : {c->fork, c->join, c->fork2, c->join2})
    if (e) cudaEventDestroy(e);
  cudaSetDevice(prev);
  delete c;
}

// Launch on stream s with programmatic stream serialization: the kernel may be
// scheduled while the kernel before it on the stream is finishing (every
// kernel of this library waits for its predecessor first, pdl_entry).
template <typename... P, typename... A>
static cudaError_t launch_pdl(void (*k)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                              A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

// The side stream and its fork / join events (created on first use).
static int ensure_side(Context* c) {
  if (!c->side) GGMS_CU(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&c->fork, &c->join, &c->fork2, &c->join2})
    if (!*e) GGMS_CU(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  return GGMS_OK;
}

// default contexts of the drop-in entry points, one per device
inline std::mutex g_default_mu;
inline Context* g_default[64];

inline int default_context(Context** out) {
  int dev = 0;
  GGMS_CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return GGMS_E_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (!g_default[dev]) {
    int rc = create_context(&g_default[dev], dev);
    if (rc != GGMS_OK) return rc;
  }
  *out = g_default[dev];
  return GGMS_OK;
}

// ------------------------------------------------------------------ workspace layout
struct Bump {
  size_t off = 0;
  size_t take(size_t bytes) {
    size_t o = (off + 255) & ~(size_t)255;
    off = o + bytes;
    return o;
  }
};


struct Plan {
  uint64_t n;
  uint32_t nk;
  uint32_t B;        // level-0 buckets
  uint32_t S;        // sample size
  uint32_t cap_seg;
  uint32_t cap_tiles;
  uint32_t ncta;     // CTAs of the two passes (identical grids)
  int assigner;
  int train_steps;
  float bound;
  float window_z;    // < 0: no PASS 1 windows
  uint64_t seed;
  uint32_t cap_q;    // batched path: caller segments with quantile bins (0: single path)
  uint32_t pl_knots; // learned PL model: requested segments (0: the default)
  uint32_t ring_st[3];  // stages of the passes' TMA rings: count, compact, coarse (0: other streams)
};


static uint32_t pow2_floor(uint64_t v) {
  uint32_t r = 1;
  while ((uint64_t)r * 2 <= v && r < (1u << 30)) r <<= 1;
  return r;
}

static int make_plan(Plan* p, uint64_t n, uint32_t nk, const ggms_opts& o) {
  p->n = n;
  p->nk = nk;
  uint32_t B = (uint32_t)o.num_buckets;
  if (B == 0) {
    // about 2^11 elements per bucket, between 2^10 and 2^13 buckets
    B = pow2_floor(std::max<uint64_t>(n >> 11, 1));
    B = std::min<uint32_t>(std::max<uint32_t>(B, 1u << 10), 1u << 13);
  }
  if (B < (1u << 10) || B > (1u << 15) || (B & (B - 1))) return GGMS_E_INVALID_ARG;
  p->B = B;
  int asg = o.assigner;
  if (asg < GGMS_ASSIGNER_AUTO || asg > GGMS_ASSIGNER_LEARNED_MLP) return GGMS_E_INVALID_ARG;
  p->assigner = asg;
  uint32_t S = (uint32_t)o.sample_size;
  if (S == 0) S = (asg == GGMS_ASSIGNER_SAMPLED) ? 1024u : (1u << 16);
  if (S < 1024u || S > 65536u || (S & (S - 1))) return GGMS_E_INVALID_ARG;
  p->S = S;
  p->ncta = 0;
  p->cap_seg = nk + 1;
  p->cap_tiles = (uint32_t)((n + TILE - 1) / TILE) + p->cap_seg;
  p->train_steps = o.train_steps > 0 ? o.train_steps : 0;
  p->bound = o.imbalance_bound > 0.0f ? o.imbalance_bound : 3.0f;
  p->window_z = o.window_z == 0.0f ? 6.0f : o.window_z;
  p->seed = o.seed;
  p->cap_q = 0;
  if (o.pl_knots != 0 && (o.pl_knots < 16 || o.pl_knots > 1024)) return GGMS_E_INVALID_ARG;
  p->pl_knots = (uint32_t)o.pl_knots;
  p->ring_st[0] = p->ring_st[1] = p->ring_st[2] = 0;
  return GGMS_OK;
}

// Options from the caller: the current layout, or the one before pl_knots was
// appended (struct_size = its offset; the new fields keep their defaults).
static int read_opts(const ggms_opts* in, ggms_opts* out) {
  ggms_default_opts(out);
  if (!in) return GGMS_OK;
  const size_t old_size = offsetof(ggms_opts, pl_knots);
  if (in->struct_size == (int32_t)sizeof(ggms_opts)) {
    *out = *in;
    out->pad0 = 0;
  } else if (in->struct_size == (int32_t)old_size) {
    memcpy(out, in, old_size);
    out->struct_size = (int32_t)sizeof(ggms_opts);
    out->pad0 = 1;  // the caller's ggms_stats ends before model_segments
  } else {
    return GGMS_E_INVALID_ARG;
  }
  return GGMS_OK;
}

static inline uint32_t float_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

// ------------------------------------------------------------------ CUDA graphs
// A call whose kernel sequence and arguments repeat (same pointers, sizes,
// options and workspace) is captured into a CUDA graph the second time it is
// seen and replayed from then on: one graph launch instead of ~30 kernel
// launches.  `enqueue(stream)` must issue only stream-ordered work (no host
// sync, no allocation).  The first call of a key runs directly, which also
// sets the kernels' attributes before any capture.  A failed capture falls
// back to running directly.
template <typename F>
static int run_graphed(Context* c, const uint64_t* key, int nkey, cudaStream_t st, F&& enqueue) {
  auto same = [&](const Context::Graph& g) {
    for (int i = 0; i < 16; ++i)
      if (g.key[i] != (i < nkey ? key[i] : 0ull)) return false;
    return true;
  };
  Context::Graph* hit = nullptr;
  for (auto& g : c->graphs)
    if (same(g)) hit = &g;
  if (hit && hit->exec) {
    hit->used = ++c->clock;
    GGMS_CU(cudaGraphLaunch(hit->exec, st));
    c->launches += hit->launches;
    ++c->graph_launches;
    return GGMS_OK;
  }
  if (!hit) {  // first sighting: remember the key (evicting the least recently used), run directly
    if (c->graphs.size() >= Context::GRAPHS) {
      auto lru = std::min_element(c->graphs.begin(), c->graphs.end(),
                                  [](const Context::Graph& a, const Context::Graph& b) { return a.used < b.used; });
      if (lru->exec) cudaGraphExecDestroy(lru->exec);
      c->graphs.erase(lru);
    }
    Context::Graph g;
    for (int i = 0; i < 16; ++i) g.key[i] = i < nkey ? key[i] : 0ull;
    g.used = ++c->clock;
    c->graphs.push_back(g);
    return enqueue(st);
  }
  // second sighting: capture, then launch
  if (!c->capture) GGMS_CU(cudaStreamCreateWithFlags(&c->capture, cudaStreamNonBlocking));
  const long long before = c->launches;
  if (cudaStreamBeginCapture(c->capture, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return enqueue(st);
  const int rc = enqueue(c->capture);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->capture, &graph);
  cudaGraphExec_t exec = nullptr;
  const bool ok = rc == GGMS_OK && e == cudaSuccess && graph &&
                  cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  const long long captured = c->launches - before;  // kernels the graph holds
  c->launches = before;
  if (!ok) {
    cudaGetLastError();
    return enqueue(st);
  }
  hit->exec = exec;
  hit->launches = captured;
  hit->used = ++c->clock;
  GGMS_CU(cudaGraphLaunch(exec, st));
  c->launches += captured;
  ++c->graph_launches;
  return GGMS_OK;
}

// Profiling slot of the current call (or null when profiling is off).
static cudaEvent_t* prof_slot(Context* c) {
  if (!c->profile) return nullptr;
  if (c->ring_count == Context::RING) return nullptr;  // ring full: drop
  int idx = (c->ring_head + c->ring_count) % Context::RING;
  if (!c->ev[idx][0])
    for (int j = 0; j < Context::NEV; ++j) cudaEventCreate(&c->ev[idx][j]);
  c->ring_count++;
  return c->ev[idx];
}
static inline void prof_rec(cudaEvent_t* slot, int j, cudaStream_t st) {
  if (slot) cudaEventRecord(slot[j], st);
}

static inline unsigned cdiv(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

// Marks the end of a call on its stream: ggms_context_status waits for it and
// then reads the status word of the call's counters (at the arena's start).
static int mark_done(Context* c, cudaStream_t st) {
  if (!c->done) GGMS_CU(cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming));
  GGMS_CU(cudaEventRecord(c->done, st));
  c->has_done = true;
  return GGMS_OK;
}


// ------------------------------------------------------------------ autotuner
// With opts->autotune set and the bucket count and pass shape left to the
// library, the first call of a shape class (type, log2 n, log2 K, assigner,
// where ks and answers live) times every candidate on the caller's own data --
// each candidate a full, correct call: 1 warm-up + 2 timed with CUDA events on
// the caller's stream -- and keeps the fastest in the context; later calls of
// the class use it.  The batched path tunes the CTAs per SM of its level
// kernels the same way (class: type, log2 n, log2 K, log2 segments).
static const Context::Tuned* tuned_find(Context* c, const uint64_t* key) {
  for (const auto& t : c->tuned)
    if (!memcmp(t.key, key, sizeof(t.key))) return &t;
  return nullptr;
}

static int bitlen64(uint64_t v) {
  int b = 0;
  while (v) { ++b; v >>= 1; }
  return b;
}

template <typename F>
static int time_calls(cudaStream_t st, F&& call, float* ms) {
  int rc = call();  // warm-up (and graph capture of repeated calls)
  if (rc) return rc;
  cudaEvent_t e0, e1;
  GGMS_CU(cudaEventCreate(&e0));
  GGMS_CU(cudaEventCreate(&e1));
  GGMS_CU(cudaEventRecord(e0, st));
  for (int i = 0; i < 2 && !rc; ++i) rc = call();
  GGMS_CU(cudaEventRecord(e1, st));
  GGMS_CU(cudaEventSynchronize(e1));
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}


}  // namespace ggms
