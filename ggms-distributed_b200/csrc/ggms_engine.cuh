// ggms_engine.cuh -- host orchestration of one call: the single-vector path
// (run_single), the batched segmented path (run_segmented), the autotuner and
// the entry-point bodies.
//
// One call = one stream-ordered sequence of kernels over a cached workspace:
// no host round trip between the passes, no allocation on the steady path,
// one H2D of the ks and one D2H of the answers when those live in host memory.
// (The reference does ~12 cudaMalloc/cudaFree and ~10 blocking copies per
// call: DistributedSMOS/bucketMultiselect.cu:583-606, 625-638, 805-845.)
//
// Each translation unit that includes this header defines GGMS_TU first and
// instantiates the templates for its own value types: the kernels (and the
// once-per-kernel attribute flags next to their launches) then belong to that
// unit alone, and the units compile in parallel.
#pragma once
#include "ggms_host.cuh"
#include "ggms_kernels.cuh"
#include "ggms_learned.cuh"
#include "ggms_window.cuh"

GGMS_BEGIN

template <typename K>
struct Workspace {
  Counters* C;
  uint32_t* kin;
  uint32_t* krank;
  uint32_t* kseg;
  uint32_t* kbin;
  K* kkey;
  K* samp_raw;
  K* samp_sorted;
  Assigner<K>* asg;       // [0] sampled, [1] learned (the PL models)
  Grid<K>* grid;          // [0] sampled, [1] learned (what the passes evaluate)
  LearnState* learn;
  Windows<K>* win;        // PASS 1 windows
  uint32_t* hist0;
  uint32_t* aflag0;
  uint32_t* kcnt0;        // per level-0 bucket: ks it holds (right after aflag0: one memset clears both)
  uint32_t* cmap0;
  uint32_t* crow;         // per-CTA bucket counts of PASS 1 -> per-CTA cursors of PASS 2
  uint32_t* ic;           // coarse mode: inclusive counts of the NGRP groups
  uint32_t* aflagc;       // coarse mode: groups holding a k
  Seg<K>* segs[2];
  uint32_t* cursor[2];
  TileRef* tiles[2];
  uint32_t* rows[2];
  uint32_t* aflag[2];
  uint32_t* khead[2];     // per segment: head of its k list (small segments)
  uint32_t* knext;        // per k: next k in its segment's list
  uint32_t* smalls;       // ids of the small segments the current level created
  uint32_t* tinies;       // ids of the tiny segments the current level created
  uint32_t* bigs[2];      // per pool: the segments a level refines (batched level 0: quantile ones)
  K* qtab;                // ... their boundaries [cap_q][QB]
  uint16_t* qdir;         // ... their directories [cap_q][QDS]
  K* points;
  K* cand[2];
  void* out_dev;
  size_t bytes;
};


template <typename K>
static Workspace<K> layout(const Plan& p, size_t out_elem_bytes, uint8_t* base) {
  Bump b;
  Workspace<K> w;
  size_t o_C = b.take(sizeof(Counters));
  size_t o_kin = b.take(4ull * p.nk);
  size_t o_krank = b.take(4ull * p.nk);
  size_t o_kseg = b.take(4ull * p.nk);
  size_t o_kbin = b.take(4ull * p.nk);
  size_t o_kkey = b.take(sizeof(K) * p.nk);
  size_t o_sr = b.take(sizeof(K) * p.S);
  size_t o_ss = b.take(sizeof(K) * p.S);
  size_t o_asg = b.take(sizeof(Assigner<K>) * 2);
  size_t o_grid = b.take(sizeof(Grid<K>) * 2);
  size_t o_learn = b.take(sizeof(LearnState));
  size_t o_win = b.take(sizeof(Windows<K>));
  size_t o_h0 = b.take(4ull * p.B);
  size_t o_a0 = b.take(4ull * (p.B / 32) + 4ull * p.B);
  size_t o_c0 = b.take(4ull * p.B);
  size_t o_crow = b.take(4ull * p.B * (p.ncta ? p.ncta : 1));
  size_t o_ic = b.take(4ull * NGRP);
  size_t o_afc = b.take(4ull * (NGRP / 32));
  size_t o_segs[2], o_cur[2], o_tiles[2], o_rows[2], o_af[2], o_cand[2], o_kh[2];
  size_t o_knext = b.take(4ull * p.nk);
  size_t o_smalls = b.take(4ull * p.cap_seg);
  size_t o_tinies = b.take(4ull * p.cap_seg);
  size_t o_bigs[2];
  for (int i = 0; i < 2; ++i) o_bigs[i] = b.take(4ull * p.cap_seg);
  size_t o_qtab = b.take(sizeof(K) * QB * p.cap_q);
  size_t o_qdir = b.take(2ull * QDS * p.cap_q);
  for (int i = 0; i < 2; ++i) {
    o_kh[i] = b.take(4ull * p.cap_seg);
    o_segs[i] = b.take(sizeof(Seg<K>) * p.cap_seg);
    o_cur[i] = b.take(4ull * p.cap_seg);
    o_tiles[i] = b.take(sizeof(TileRef) * p.cap_tiles);
    o_rows[i] = b.take(4ull * NBIN * p.cap_seg);
    o_af[i] = b.take(4ull * NBIN_WORDS * p.cap_seg);
  }
  size_t o_pts = b.take(sizeof(K) * p.nk);
  for (int i = 0; i < 2; ++i) o_cand[i] = b.take(sizeof(K) * p.n);
  size_t o_out = b.take(out_elem_bytes * p.nk);
  w.bytes = b.take(0) + 256;
  if (!base) return w;
  w.C = (Counters*)(base + o_C);
  w.kin = (uint32_t*)(base + o_kin);
  w.krank = (uint32_t*)(base + o_krank);
  w.kseg = (uint32_t*)(base + o_kseg);
  w.kbin = (uint32_t*)(base + o_kbin);
  w.kkey = (K*)(base + o_kkey);
  w.samp_raw = (K*)(base + o_sr);
  w.samp_sorted = (K*)(base + o_ss);
  w.asg = (Assigner<K>*)(base + o_asg);
  w.grid = (Grid<K>*)(base + o_grid);
  w.learn = (LearnState*)(base + o_learn);
  w.win = (Windows<K>*)(base + o_win);
  w.hist0 = (uint32_t*)(base + o_h0);
  w.aflag0 = (uint32_t*)(base + o_a0);
  w.kcnt0 = w.aflag0 + p.B / 32;
  w.cmap0 = (uint32_t*)(base + o_c0);
  w.crow = (uint32_t*)(base + o_crow);
  w.ic = (uint32_t*)(base + o_ic);
  w.aflagc = (uint32_t*)(base + o_afc);
  for (int i = 0; i < 2; ++i) {
    w.segs[i] = (Seg<K>*)(base + o_segs[i]);
    w.cursor[i] = (uint32_t*)(base + o_cur[i]);
    w.tiles[i] = (TileRef*)(base + o_tiles[i]);
    w.rows[i] = (uint32_t*)(base + o_rows[i]);
    w.aflag[i] = (uint32_t*)(base + o_af[i]);
    w.cand[i] = (K*)(base + o_cand[i]);
    w.khead[i] = (uint32_t*)(base + o_kh[i]);
  }
  w.knext = (uint32_t*)(base + o_knext);
  w.smalls = (uint32_t*)(base + o_smalls);
  w.tinies = (uint32_t*)(base + o_tinies);
  for (int i = 0; i < 2; ++i) w.bigs[i] = (uint32_t*)(base + o_bigs[i]);
  w.qtab = (K*)(base + o_qtab);
  w.qdir = (uint16_t*)(base + o_qdir);
  w.points = (K*)(base + o_pts);
  w.out_dev = (void*)(base + o_out);
  return w;
}


// The refinement levels first..maxlev (1-based) of the single-vector path.
// Captured into a graph, level l becomes an IF node and level l + 1 is nested
// inside its body, so a level without segments skips every later level at
// the cost of one conditional node.  The condition of the first level is set
// by an earlier kernel (handle `first`, created by level_handle()); the later
// ones by lvl_gate at the end of the enclosing level.  Run directly, the
// levels' kernels are launched as they are (each returns at once when there
// is no work).  body(stream, l) enqueues level l's kernels.
static int level_handle(cudaStream_t s, cudaGraphConditionalHandle* h) {
  *h = 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  GGMS_CU(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusActive) return GGMS_OK;
  cudaGraph_t g = nullptr;
  GGMS_CU(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr));
  GGMS_CU(cudaGraphConditionalHandleCreate(h, g, 0u, cudaGraphCondAssignDefault));
  return GGMS_OK;
}

template <typename F>
static int enqueue_levels(Context* c, cudaStream_t s, Counters* C, int l, int maxlev,
                          cudaGraphConditionalHandle first, F&& body) {
  if (l > maxlev) return GGMS_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  GGMS_CU(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusActive) {
    const int rc = body(s, l);
    if (rc) return rc;
    return enqueue_levels(c, s, C, l + 1, maxlev, 0, body);
  }
  if (l > Context::MAX_NEST) return GGMS_E_INTERNAL;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  cudaGraphConditionalHandle h = first;
  if (!h) {
    GGMS_CU(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    GGMS_CU(cudaGraphConditionalHandleCreate(&h, g, 0u, cudaGraphCondAssignDefault));
    ++c->launches;
    lvl_gate<<<1, 1, 0, s>>>(C, l & 1, h);
  }
  GGMS_CU(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeIf;
  np.conditional.size = 1;
  cudaGraphNode_t cn;
  GGMS_CU(cudaGraphAddNode(&cn, g, deps, nd, &np));
  cudaStream_t& bs = c->bodies[l - 1];
  if (!bs) GGMS_CU(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
  GGMS_CU(cudaStreamBeginCaptureToGraph(bs, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
  int rc = body(bs, l);
  if (!rc) rc = enqueue_levels(c, bs, C, l + 1, maxlev, 0, body);
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(bs, &out);
  if (rc) return rc;
  GGMS_CU(e);
  GGMS_CU(cudaStreamUpdateCaptureDependencies(s, &cn, 1, cudaStreamSetCaptureDependencies));
  return GGMS_OK;
}

// ------------------------------------------------------------------ kernel configs
constexpr int LV_NT = 256;
constexpr int MAX_LEVELS_32 = 3;
constexpr int MAX_LEVELS_64 = 6;

template <typename T>
static size_t l0_count_smem(uint32_t B, int nt, int unroll, uint32_t nst) {
  const size_t base = GRID_SMEM + (size_t)B * 4u + wq_bytes((uint32_t)nt, sizeof(typename KeyOf<T>::K));
  return unroll < 0 ? ((base + 127) & ~(size_t)127) + ring_bytes(unroll, nst) : base;
}
template <typename T>
static size_t l0_coarse_smem(int nt, int unroll, uint32_t nst) {
  const size_t ch = (size_t)nt * coarse_du(unroll < 0 ? 0 : unroll) * (16 / sizeof(T));
  const size_t base = GRID_SMEM + ch * (sizeof(typename KeyOf<T>::K) + 1);
  return unroll < 0 ? ((base + 127) & ~(size_t)127) + ring_bytes(unroll, nst) : base;
}
template <typename T>
static size_t l0_compact_smem(uint32_t B, int nt, int unroll, uint32_t nst) {
  const size_t base = GRID_SMEM +
                      (MAX_B0 / 32 + l0_compact_qwords((uint32_t)nt, sizeof(typename KeyOf<T>::K)) + HOT_WORDS) * 4u +
                      (size_t)B * 4u;
  return unroll < 0 ? ((base + 127) & ~(size_t)127) + ring_bytes(unroll, nst) : base;
}

// Launch shapes of the two passes: CTA size x 16-byte loads in flight per
// thread (unroll 2, 4 or 8, register streams), unroll -1: the TMA ring (bulk
// copies into shared-memory stages), unroll -2: per-thread async copies into
// shared memory; the default and the autotuner pick among these instantiations.
template <typename T>
struct PassVariant {
  using K = typename KeyOf<T>::K;
  int nt, unroll;
  void (*count)(const T*, uint64_t, const Grid<K>*, Counters*, const Windows<K>*, uint32_t*, uint32_t*, uint32_t);
  void (*compact)(const T*, uint64_t, const Grid<K>*, Counters*, const Windows<K>*, const uint32_t*,
                  const uint32_t*, K*, uint64_t, uint32_t, const uint32_t*);
  void (*coarse)(const T*, uint64_t, const Grid<K>*, Counters*, const uint32_t*, const uint32_t*, K*, uint64_t,
                 uint32_t);
};

template <typename T>
static const PassVariant<T>* pass_variant(int nt, int unroll) {
  static const PassVariant<T> v[] = {
      {256, 4, l0_count<T, 256, 4>, l0_compact<T, 256, 4>, l0_compact_coarse<T, 256, 4>},
      {256, 8, l0_count<T, 256, 8>, l0_compact<T, 256, 8>, l0_compact_coarse<T, 256, 8>},
      {512, 2, l0_count<T, 512, 2>, l0_compact<T, 512, 2>, l0_compact_coarse<T, 512, 2>},
      {512, 4, l0_count<T, 512, 4>, l0_compact<T, 512, 4>, l0_compact_coarse<T, 512, 4>},
      {512, 8, l0_count<T, 512, 8>, l0_compact<T, 512, 8>, l0_compact_coarse<T, 512, 8>},
      {1024, 2, l0_count<T, 1024, 2>, l0_compact<T, 1024, 2>, l0_compact_coarse<T, 1024, 2>},
      {1024, 4, l0_count<T, 1024, 4>, l0_compact<T, 1024, 4>, l0_compact_coarse<T, 1024, 4>},
      {1024, -1, l0_count<T, 1024, -1>, l0_compact<T, 1024, -1>, l0_compact_coarse<T, 1024, -1>},
      {1024, -2, l0_count<T, 1024, -2>, l0_compact<T, 1024, -2>, l0_compact_coarse<T, 1024, -2>},
  };
  for (const auto& x : v)
    if (x.nt == nt && x.unroll == unroll) return &x;
  return nullptr;
}

constexpr int DEFAULT_PASS_NT = 1024;
constexpr int DEFAULT_PASS_UNROLL = 4;  // register streams (the staged ones measure no faster here)

// Stages of the TMA ring of one pass kernel whose other shared memory is
// `base` bytes: as many 32 KB stages (2..4) as fit next to it in what a CTA
// may use (its static shared memory included, with margin).
static uint32_t ring_stages(Context* c, size_t base) {
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device) != cudaSuccess)
    optin = 227 * 1024;
  const size_t margin = 8192 + 128;  // static shared memory of the pass kernels, alignment
  const size_t room = (size_t)optin > base + margin ? (size_t)optin - base - margin : 0;
  return (uint32_t)std::min<size_t>(4, std::max<size_t>(2, room / RING_BYTES));
}

// Stages of the three pass kernels' rings: [0] count, [1] compact, [2] coarse
// (0 for the other streams).
template <typename T>
static void pass_stages(Context* c, const PassVariant<T>* pv, uint32_t B, uint32_t* st) {
  for (int i = 0; i < 3; ++i) st[i] = 0u;
  if (pv->unroll != -1) return;
  st[0] = ring_stages(c, l0_count_smem<T>(B, pv->nt, -1, 0));
  st[1] = ring_stages(c, l0_compact_smem<T>(B, pv->nt, -1, 0));
  st[2] = ring_stages(c, l0_coarse_smem<T>(pv->nt, -1, 0));
}

// The two passes must split the input among CTAs identically (PASS 2 writes
// into per-CTA ranges sized by PASS 1), so both get the same grid: as many
// CTAs as fit on every SM at once for the larger of the two.
template <typename T>
static int l0_ncta(Context* c, const PassVariant<T>* pv, uint32_t B, const uint32_t* nst, uint32_t* ncta) {
  const size_t s1 = l0_count_smem<T>(B, pv->nt, pv->unroll, nst[0]);
  const size_t s2 = l0_compact_smem<T>(B, pv->nt, pv->unroll, nst[1]);
  const size_t s3 = l0_coarse_smem<T>(pv->nt, pv->unroll, nst[2]);
  GGMS_CU(cudaFuncSetAttribute((const void*)pv->count, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1));
  GGMS_CU(cudaFuncSetAttribute((const void*)pv->compact, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2));
  GGMS_CU(cudaFuncSetAttribute((const void*)pv->coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s3));
  int o1 = 0, o2 = 0, o3 = 0;
  GGMS_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, (const void*)pv->count, pv->nt, s1));
  GGMS_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, (const void*)pv->compact, pv->nt, s2));
  GGMS_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o3, (const void*)pv->coarse, pv->nt, s3));
  *ncta = (uint32_t)(std::max(1, std::min(std::min(o1, o2), o3)) * c->sms);
  return GGMS_OK;
}

// Up to this many ks, the steps between the passes run in one CTA (l0_between).
constexpr uint32_t L0_FUSED_MAX_KS = 65536;

template <typename K>
static int setup_attrs() {
  static bool done = false;
  if (done) return GGMS_OK;
  GGMS_CU(cudaFuncSetAttribute(l0_between<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)l0_between_smem(MAX_B0)));
  GGMS_CU(cudaFuncSetAttribute(l0_scan<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(4u * MAX_B0)));
  GGMS_CU(cudaFuncSetAttribute(setup_sampled<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(SetupSmem<K>)));
  GGMS_CU(cudaFuncSetAttribute(l0_window<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)l0_window_smem<K>(MAX_B0)));
  done = true;
  return GGMS_OK;
}

constexpr int SS_NT = 512;

template <typename InT, typename K = typename KeyOf<InT>::K>
static int launch_small_select(Context* ctx, const InT* src, const Seg<K>* segs_q, const uint32_t* khead_q,
                               const Workspace<K>& w, const Caps& caps, cudaStream_t st,
                               const int64_t* k_off = nullptr) {
  static bool attr = false;
  const size_t sm = SMALL_SMEM + (size_t)SS_GROUP * 256 * 4;
  if (!attr) {
    GGMS_CU(cudaFuncSetAttribute(small_select<InT, SS_NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sm));
    attr = true;
  }
  ++ctx->launches;
  GGMS_CU(launch_pdl(small_select<InT, SS_NT>, ctx->sms * 2, SS_NT, sm, st, src, segs_q, w.smalls, w.C, khead_q,
                     w.knext, k_off, w.krank, w.kseg, w.kkey, caps.small_keys, caps));
  // the warp finisher (its own list of segments) runs beside the CTA finisher:
  // it does not wait for it before its work (tiny_select)
  if (caps.tiny_keys) {
    ++ctx->launches;
    GGMS_CU(launch_pdl(tiny_select<InT, TS_NT>, ctx->sms * 8, TS_NT, 0, st, src, segs_q, w.tinies, w.C, khead_q,
                       w.knext, k_off, w.krank, w.kseg, w.kkey, caps));
  }
  return GGMS_OK;
}

// Profiling slot of the current call (or null when profiling is off).

// ------------------------------------------------------------------ the single-vector path

// The sample sort's cluster: attributes set once per key type; 16 CTAs when the
// sample has at least one key per thread of 16 CTAs and the device can place a
// 16-CTA cluster of this kernel, else 8; 0: too small for a cluster (S < 8192);
// -1: the attributes could not be set.
template <typename K, int CTAS>
static cudaError_t launch_sort_cluster(cudaStream_t s, const K* drawn, uint32_t S, K* sorted) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CTAS);
  cfg.blockDim = dim3(CS_NT);
  cfg.dynamicSmemBytes = sizeof(ClusterSortSmem<K, CTAS>);
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CTAS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  return cudaLaunchKernelEx(&cfg, asg_sort_cluster<K, CTAS>, drawn, S, sorted);
}

template <typename K>
static int sort_cluster_ctas(uint32_t S) {
  static int have16 = -1;  // -1: not probed yet
  if (have16 < 0) {
    have16 = 0;
    if (cudaFuncSetAttribute(asg_sort_cluster<K, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(ClusterSortSmem<K, 8>)) != cudaSuccess ||
        cudaFuncSetAttribute(asg_sort_cluster<K, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(ClusterSortSmem<K, 16>)) != cudaSuccess)
      return -1;
    if (cudaFuncSetAttribute(asg_sort_cluster<K, 16>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
        cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(16);
      cfg.blockDim = dim3(CS_NT);
      cfg.dynamicSmemBytes = sizeof(ClusterSortSmem<K, 16>);
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = 16;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int nclusters = 0;
      if (cudaOccupancyMaxActiveClusters(&nclusters, asg_sort_cluster<K, 16>, &cfg) == cudaSuccess &&
          nclusters >= 1)
        have16 = 1;
    }
    cudaGetLastError();  // a refused probe leaves no error behind
  }
  if (S >= cs_min_s(16) && have16) return 16;
  return S >= cs_min_s(8) ? 8 : 0;
}

template <typename T>
static int run_single(Context* ctx, const T* d_in, uint64_t n, const uint32_t* ks, uint64_t nk64,
                      T* out, const ggms_opts& o_in, cudaStream_t st, bool topk = false) {
  using K = typename KeyOf<T>::K;
  if (!d_in || n == 0 || n > 0xFFFFFFFFull || nk64 > 0x7FFFFFFFull) return GGMS_E_INVALID_ARG;
  if (nk64 == 0) return GGMS_OK;
  if ((!ks && !topk) || !out) return GGMS_E_INVALID_ARG;
  if (topk && nk64 > n) return GGMS_E_INVALID_ARG;
  ggms_opts o = o_in;
  if (topk) o.ks_on_device = 1;  // no k array to upload
  if ((uintptr_t)d_in % sizeof(T) != 0) return GGMS_E_INVALID_ARG;
  const uint32_t nk = (uint32_t)nk64;
  if (!o.ks_on_device) {
    for (uint32_t i = 0; i < nk; ++i)
      if (ks[i] < 1u || (uint64_t)ks[i] > n) return GGMS_E_INVALID_ARG;
  }
  Plan p;
  int rc = make_plan(&p, n, nk, o);
  if (rc) return rc;
  GGMS_CU(cudaSetDevice(ctx->device));
  const PassVariant<T>* pv = pass_variant<T>(o.pass_threads ? o.pass_threads : DEFAULT_PASS_NT,
                                              o.pass_unroll ? o.pass_unroll : DEFAULT_PASS_UNROLL);
  if (!pv) return GGMS_E_INVALID_ARG;
  pass_stages<T>(ctx, pv, p.B, p.ring_st);
  rc = l0_ncta<T>(ctx, pv, p.B, p.ring_st, &p.ncta);
  if (rc) return rc;
  Workspace<K> w0 = layout<K>(p, sizeof(T), nullptr);
  rc = ensure_arena(ctx, w0.bytes);
  if (rc) return rc;
  Workspace<K> w = layout<K>(p, sizeof(T), ctx->arena);
  const bool host_k = !o.ks_on_device && !topk, host_out = !o.out_on_device;
  const size_t pin_bytes = (host_k ? 4ull * nk : 0) + (host_out ? sizeof(T) * nk : 0) + sizeof(Counters) + 64;
  rc = ensure_pinned(ctx, pin_bytes);
  if (rc) return rc;
  uint8_t* pin = ctx->pinned;
  Counters* pin_C = (Counters*)pin;
  uint8_t* pin_k = pin + ((sizeof(Counters) + 63) & ~(size_t)63);
  uint8_t* pin_out = pin_k + (host_k ? ((4ull * nk + 63) & ~(size_t)63) : 0);

  const Caps caps{p.cap_seg, p.cap_tiles, p.nk, (uint32_t)(SMALL_SMEM / sizeof(K)), 0u};
  if (host_k && !topk) {
    // host side, every call: the previous call's upload from the same pinned
    // buffer may still be queued (calls with device-resident answers return
    // without a sync), so wait for it first
    if (ctx->pin_busy) GGMS_CU(cudaEventSynchronize(ctx->pin_busy));
    memcpy(pin_k, ks, 4ull * nk);
  }
  cudaEvent_t* prof = prof_slot(ctx);
  // the stream-ordered part: captured once and replayed when the call repeats
  auto enqueue = [&](cudaStream_t s) -> int {
    prof_rec(prof, 0, s);
    GGMS_CU(cudaMemsetAsync(w.C, 0, sizeof(Counters), s));
    const uint32_t* d_k = ks;
    if (host_k && !topk) {
      GGMS_CU(cudaMemcpyAsync(w.kin, pin_k, 4ull * nk, cudaMemcpyHostToDevice, s));
      d_k = w.kin;
    }
    ++ctx->launches;
    if (topk)
      k_init_topk<<<cdiv(nk, 256), 256, 0, s>>>(nk, n, w.krank, w.kseg);
    else
      k_init_single<<<cdiv(nk, 256), 256, 0, s>>>(d_k, nk, n, w.krank, w.kseg, w.C);

    // ---- level-0 assigner
    const uint32_t S = p.S;
    const int cs_ctas = sort_cluster_ctas<K>(S);
    if (cs_ctas < 0) return GGMS_E_CUDA;
    if (cs_ctas) {  // draw the sample over the whole GPU, sort it in one cluster
      ctx->launches += 2;
      GGMS_CU(launch_pdl(asg_sample<T>, cdiv(S, 256), 256, 0, s, d_in, n, S, p.seed, w.samp_raw));
      const cudaError_t e_sort = cs_ctas == 16 ? launch_sort_cluster<K, 16>(s, w.samp_raw, S, w.samp_sorted)
                                               : launch_sort_cluster<K, 8>(s, w.samp_raw, S, w.samp_sorted);
      GGMS_CU(e_sort);
    } else {  // up to 4096 keys: draw them, then one CTA sorts them
      ctx->launches += 2;
      asg_sample<T><<<cdiv(S, 256), 256, 0, s>>>(d_in, n, S, p.seed, w.samp_raw);
      if (S <= 1024)
        asg_sort_chunks<K, 1024, 1024><<<1, 1024, 0, s>>>(w.samp_raw, w.samp_sorted, S);
      else if (S <= 2048)
        asg_sort_chunks<K, 2048, 1024><<<1, 1024, 0, s>>>(w.samp_raw, w.samp_sorted, S);
      else
        asg_sort_chunks<K, 4096, 1024><<<1, 1024, 0, s>>>(w.samp_raw, w.samp_sorted, S);
    }
    prof_rec(prof, 6, s);
    rc = setup_attrs<K>();
    if (rc) return rc;
    if (p.assigner == GGMS_ASSIGNER_SAMPLED) {
      ++ctx->launches;
      GGMS_CU(launch_pdl(setup_sampled<K>, 1, SETUP_NT, sizeof(SetupSmem<K>), s, w.samp_sorted, S, p.B, &w.asg[0],
                         &w.grid[0]));
    } else {
      // the sampled grid (fallback and judge) is built on a side stream while
      // the learned model's knots and statistics are computed: fork and join
      if (const int r_ = ensure_side(ctx)) return r_;
      GGMS_CU(cudaEventRecord(ctx->fork, s));
      GGMS_CU(cudaStreamWaitEvent(ctx->side, ctx->fork, 0));
      ++ctx->launches;
      setup_sampled<K><<<1, SETUP_NT, sizeof(SetupSmem<K>), ctx->side>>>(w.samp_sorted, S, p.B, &w.asg[0],
                                                                           &w.grid[0]);
      GGMS_CU(cudaEventRecord(ctx->join, ctx->side));
      rc = learn_and_choose<K>(p.assigner, w.samp_sorted, S, p.B, p.train_steps, p.bound, w.asg,
                               w.grid, w.learn, &w.C->asg_choice, w.krank, nk, n, p.window_z, s,
                               &ctx->launches, ctx->join, p.pl_knots);
      if (rc) return rc;
    }

    // ---- PASS 1 windows
    prof_rec(prof, 7, s);
    const bool windows = p.window_z >= 0.0f;
    if (windows) {
      ++ctx->launches;
      GGMS_CU(launch_pdl(l0_window<K>, 1, WIN_NT, l0_window_smem<K>(p.B), s, w.samp_sorted, S, w.krank, nk, n,
                         w.grid, w.C, p.window_z, w.win));
    }

    // ---- PASS 1: count
    const int grid_c = (int)p.ncta;
    // the histogram, the flags and k counts (and, without windows, the windows)
    static_assert(sizeof(Windows<K>) % 4 == 0, "zeroed as words");
    ++ctx->launches;
    GGMS_CU(launch_pdl(zero_words, 8, 1024, 0, s, w.hist0, p.B, w.aflag0, p.B / 32 + p.B,
                       windows ? (uint32_t*)nullptr : (uint32_t*)w.win, (uint32_t)(sizeof(Windows<K>) / 4)));
    prof_rec(prof, 1, s);
    ++ctx->launches;
    GGMS_CU(launch_pdl(pv->count, grid_c, pv->nt, l0_count_smem<T>(p.B, pv->nt, pv->unroll, p.ring_st[0]), s, d_in,
                       n, w.grid, w.C, w.win, w.hist0, w.crow, p.ring_st[0]));
    prof_rec(prof, 2, s);
    if (nk <= L0_FUSED_MAX_KS) {
      // scan, locate and the coarse-mode decision in one CTA
      ++ctx->launches;
      GGMS_CU(launch_pdl(l0_between<K>, 1, 1024, l0_between_smem(p.B), s, w.hist0, p.B, w.C, w.win, nk, w.krank,
                         w.kseg, w.kbin, w.kcnt0, w.aflag0, w.ic, w.aflagc));
    } else {
      ++ctx->launches;
      l0_scan<K><<<1, 1024, 4u * p.B, s>>>(w.hist0, p.B, w.C, w.win, w.aflagc);
      ++ctx->launches;
      lvl_locate_rows<<<cdiv(nk, 256), 256, 0, s>>>(w.hist0, p.B, nk, w.krank, w.kseg, w.kbin,
                                                       w.aflag0, p.B / 32, w.C, w.kcnt0);
      // most buckets hold a k: copy groups of buckets instead (coarse mode)
      ++ctx->launches;
      l0_mode_ks<K><<<cdiv(nk, 256), 256, 0, s>>>(w.hist0, w.aflag0, p.B, w.win, w.C, w.ic, w.aflagc, nk, w.krank,
                                                   w.kseg, w.kbin);
    }
    ++ctx->launches;
    GGMS_CU(launch_pdl(l0_children<K>, cdiv(p.B, 256), 256, 0, s, w.hist0, w.aflag0, p.B, w.grid, w.C, w.win,
                       w.cmap0, w.segs[1], w.cursor[1], w.tiles[1], w.points, w.khead[1], w.smalls, w.bigs[1], caps,
                       w.ic, w.aflagc, w.kcnt0, tiny_keys<K>(), w.tinies));
    // the first refinement level runs only when a level-0 child needs it: the
    // kernel that relabels the ks after l0_children sets that condition
    cudaGraphConditionalHandle lev1 = 0;
    rc = level_handle(s, &lev1);
    if (rc) return rc;
    ++ctx->launches;
    GGMS_CU(launch_pdl(l0_relabel_bases<K>, ctx->sms * 4, 256, 0, s, w.cmap0, nk, w.kbin, w.kseg, w.kkey, w.points,
                       w.C, w.segs[1], w.khead[1], w.knext, w.crow, p.B, p.ncta, caps, lev1));
    // ---- PASS 2: compact the buckets that still need refinement
    prof_rec(prof, 3, s);
    ++ctx->launches;
    GGMS_CU(launch_pdl(pv->compact, grid_c, pv->nt, l0_compact_smem<T>(p.B, pv->nt, pv->unroll, p.ring_st[1]), s,
                       d_in, n, w.grid, w.C, w.win, w.cmap0, w.crow, w.cand[0], (uint64_t)n, p.ring_st[1],
                       w.hist0));
    ++ctx->launches;  // one of the two PASS-2 kernels returns at once
    GGMS_CU(launch_pdl(pv->coarse, grid_c, pv->nt, l0_coarse_smem<T>(pv->nt, pv->unroll, p.ring_st[2]), s, d_in,
                       n, w.grid, w.C, w.cmap0, w.crow, w.cand[0], (uint64_t)n, p.ring_st[2]));
    prof_rec(prof, 4, s);
    {
      // level 0 also has warp-sized children (l0_children); the refinement
      // levels of this path do not
      Caps c0 = caps;
      c0.tiny_keys = tiny_keys<K>();
      rc = launch_small_select<K>(ctx, w.cand[0], w.segs[1], w.khead[1], w, c0, s);
    }
    if (rc) return rc;

    // ---- refinement levels over candidates
    const int maxlev = (sizeof(K) == 4) ? MAX_LEVELS_32 : MAX_LEVELS_64;
    const int lv_grid = ctx->sms * 8;
    const int seg_grid = std::min<int>((int)p.cap_seg, ctx->sms * 2);
    rc = enqueue_levels(ctx, s, w.C, 1, maxlev, lev1, [&](cudaStream_t s, int l) -> int {
      const int pp = l & 1, q = pp ^ 1;
      const K* src = w.cand[(l - 1) & 1];
      K* dst = w.cand[l & 1];
      ++ctx->launches;
      lvl_prep<<<ctx->sms * 2, 256, 0, s>>>(w.rows[pp], w.aflag[pp], w.bigs[pp], w.C, pp, caps);
      ++ctx->launches;
      lvl_count<K, LV_NT><<<lv_grid, LV_NT, 0, s>>>(src, w.segs[pp], w.tiles[pp], w.C, pp, w.rows[pp], caps,
                                                     nullptr, nullptr);
      ++ctx->launches;
      lvl_scan<<<seg_grid, 1024, 0, s>>>(w.rows[pp], w.bigs[pp], w.C, pp, caps);
      ++ctx->launches;
      lvl_locate_rows<<<cdiv(nk, 256), 256, 0, s>>>(w.rows[pp], NBIN, nk, w.krank, w.kseg, w.kbin,
                                                       w.aflag[pp], NBIN_WORDS, w.C);
      ++ctx->launches;
      lvl_children<K, 1024><<<seg_grid, 1024, 0, s>>>(w.rows[pp], w.aflag[pp], w.segs[pp], w.C, pp,
                                                       w.segs[q], w.cursor[q], w.tiles[q], w.points,
                                                       w.khead[q], w.smalls, w.tinies, w.bigs[pp],
                                                       w.bigs[q], caps, nullptr);
      ++ctx->launches;
      lvl_relabel<K><<<cdiv(nk, 256), 256, 0, s>>>(w.rows[pp], NBIN, nk, w.kbin, w.kseg, w.kkey,
                                                      w.points, w.C, w.segs[q], w.khead[q], w.knext);
      if (l < maxlev) {
        ++ctx->launches;
        lvl_compact<K, LV_NT><<<lv_grid, LV_NT, 0, s>>>(src, w.segs[pp], w.tiles[pp], w.C, pp,
                                                         w.rows[pp], w.segs[q], w.cursor[q], dst, caps,
                                                         nullptr, nullptr);
        return launch_small_select<K>(ctx, dst, w.segs[q], w.khead[q], w, caps, s);
      }
      return GGMS_OK;
    });
    if (rc) return rc;

    // ---- answers
    prof_rec(prof, 8, s);
    T* d_out = host_out ? (T*)w.out_dev : out;
    ++ctx->launches;
    write_out<T><<<cdiv(nk, 256), 256, 0, s>>>(w.kkey, w.kseg, nk, d_out, w.C);
    if (cudaGetLastError() != cudaSuccess) return GGMS_E_CUDA;
    if (host_out) GGMS_CU(cudaMemcpyAsync(pin_out, d_out, sizeof(T) * nk, cudaMemcpyDeviceToHost, s));
    if (host_out || o.stats) GGMS_CU(cudaMemcpyAsync(pin_C, w.C, sizeof(Counters), cudaMemcpyDeviceToHost, s));
    prof_rec(prof, 5, s);
    return GGMS_OK;
  };
  if (o.stats || prof) {
    rc = enqueue(st);
  } else {
    const uint64_t key[] = {0x51Eull + sizeof(T) + (topk ? 256u : 0u) + (std::is_signed<T>::value ? 16u : 0u) +
                                (std::is_floating_point<T>::value ? 32u : 0u),
                            (uint64_t)(uintptr_t)d_in, n, host_k ? 1ull : (uint64_t)(uintptr_t)ks, nk,
                            host_out ? 1ull : (uint64_t)(uintptr_t)out,
                            (uint64_t)p.assigner | ((uint64_t)p.B << 8) | ((uint64_t)p.S << 24),
                            p.seed, (uint64_t)(uint32_t)p.train_steps | ((uint64_t)pv->nt << 32),
                            (uint64_t)pv->unroll | ((uint64_t)float_bits(p.bound) << 8),
                            (uint64_t)float_bits(p.window_z), (uint64_t)(uintptr_t)ctx->arena,
                            (uint64_t)(uintptr_t)ctx->pinned, (uint64_t)p.pl_knots};
    rc = run_graphed(ctx, key, (int)(sizeof(key) / sizeof(key[0])), st, enqueue);
  }
  if (rc) return rc;
  rc = mark_done(ctx, st);
  if (rc) return rc;
  if (host_k && !topk) {
    if (!ctx->pin_busy) GGMS_CU(cudaEventCreateWithFlags(&ctx->pin_busy, cudaEventDisableTiming));
    GGMS_CU(cudaEventRecord(ctx->pin_busy, st));
  }
  const bool need_sync = host_out || o.stats;
  if (!need_sync) return GGMS_OK;
  GGMS_CU(cudaStreamSynchronize(st));
  if (host_out) memcpy(out, pin_out, sizeof(T) * nk);
  if (o.stats) {
    ggms_stats* s = o.stats;
    Grid<K> a_used;
    GGMS_CU(cudaMemcpy(&a_used, &w.grid[pin_C->asg_choice], sizeof(Grid<K>), cudaMemcpyDeviceToHost));
    LearnState ls;
    GGMS_CU(cudaMemcpy(&ls, w.learn, sizeof(LearnState), cudaMemcpyDeviceToHost));
    s->assigner_used = (int32_t)a_used.kind;
    s->num_buckets = (int32_t)p.B;
    s->full_passes = (int32_t)pin_C->passes;
    s->levels = (int32_t)pin_C->levels_run;
    s->candidates = (int64_t)pin_C->cand0;
    s->refine_elements = (int64_t)pin_C->refine_elems;
    s->active_buckets = (int32_t)pin_C->active0;
    s->point_buckets = (int32_t)pin_C->point0;
    s->small_segments = (int32_t)pin_C->small_segs;
    s->sample_size = (int32_t)p.S;
    s->bucket_max_over_mean = (float)pin_C->max_bucket0 / ((float)n / (float)p.B);
    s->model_imbalance = (p.assigner == GGMS_ASSIGNER_SAMPLED) ? 0.0f : ls.imbalance;
    s->model_loss = p.assigner == GGMS_ASSIGNER_SAMPLED        ? 0.0f
                    : p.assigner == GGMS_ASSIGNER_LEARNED_MLP ? ls.mlp_loss
                                                              : ls.loss;
    s->window_runs = (int32_t)pin_C->win_runs;
    if (!o.pad0) s->model_segments = (p.assigner == GGMS_ASSIGNER_SAMPLED || a_used.kind == GGMS_ASSIGNER_SAMPLED)
                                         ? 0 : (int32_t)ls.M;
  }
  if (pin_C->status) return (int)pin_C->status;
  return GGMS_OK;
}


template <typename T>
static int run_single_tuned(Context* c, const T* d_in, uint64_t n, const uint32_t* ks, uint64_t nk, T* out,
                            const ggms_opts& o, cudaStream_t st, bool topk = false) {
  if (!o.autotune || o.num_buckets || o.pass_threads || o.pass_unroll || n == 0 || nk == 0)
    return run_single<T>(c, d_in, n, ks, nk, out, o, st, topk);
  const uint64_t key[4] = {sizeof(T) | (std::is_signed<T>::value ? 16u : 0u) |
                               (std::is_floating_point<T>::value ? 32u : 0u) | (topk ? 64u : 0u),
                           (uint64_t)bitlen64(n) | ((uint64_t)bitlen64(nk) << 8),
                           (uint64_t)o.assigner | ((uint64_t)o.ks_on_device << 8) | ((uint64_t)o.out_on_device << 9),
                           (uint64_t)float_bits(o.window_z)};
  ggms_opts b = o;
  b.autotune = 0;
  if (const Context::Tuned* t = tuned_find(c, key)) {
    b.num_buckets = t->B;
    b.pass_threads = t->nt;
    b.pass_unroll = t->unroll;
    return run_single<T>(c, d_in, n, ks, nk, out, b, st, topk);
  }
  static const int Bs[] = {4096, 8192, 16384};
  static const int shapes[][2] = {{1024, 4}, {1024, -2}, {512, 4}, {512, 8}};
  float best = 3.4e38f;
  Context::Tuned pick{{key[0], key[1], key[2], key[3]}, 8192, DEFAULT_PASS_NT, DEFAULT_PASS_UNROLL, 8};
  for (int B : Bs) {
    for (const auto& sh : shapes) {
      ggms_opts t = b;
      t.num_buckets = B;
      t.pass_threads = sh[0];
      t.pass_unroll = sh[1];
      float ms = 0.0f;
      const int rc = time_calls(st, [&] { return run_single<T>(c, d_in, n, ks, nk, out, t, st, topk); }, &ms);
      if (rc) return rc;
      if (ms < best) {
        best = ms;
        pick.B = B;
        pick.nt = sh[0];
        pick.unroll = sh[1];
      }
    }
  }
  c->tuned.push_back(pick);
  b.num_buckets = pick.B;
  b.pass_threads = pick.nt;
  b.pass_unroll = pick.unroll;
  return run_single<T>(c, d_in, n, ks, nk, out, b, st, topk);
}

template <typename T>
static int dropin(const T* d_vector, int length, const uint32_t* kVals, int numKs, T* outputs) {
  if (length <= 0 || numKs < 0) return GGMS_E_INVALID_ARG;
  Context* c = nullptr;
  int rc = default_context(&c);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(c->mu);
  ggms_opts o;
  ggms_default_opts(&o);
  return run_single<T>(c, d_vector, (uint64_t)length, kVals, (uint64_t)numKs, outputs, o, 0);
}

template <typename T>
static int topk_call(ggms_context* cx, const T* d_in, int64_t n, int64_t K, T* out,
                     const ggms_opts* opts, void* stream) {
  if (n <= 0 || K <= 0) return GGMS_E_INVALID_ARG;
  ggms_opts o;
  if (read_opts(opts, &o) != GGMS_OK) return GGMS_E_INVALID_ARG;
  Context* c = (Context*)cx;
  if (!c) {
    int rc = default_context(&c);
    if (rc) return rc;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  return run_single_tuned<T>(c, d_in, (uint64_t)n, nullptr, (uint64_t)K, out, o, (cudaStream_t)stream, true);
}

template <typename T>
static int ex(ggms_context* cx, const T* d_in, int64_t n, const uint32_t* ks, int64_t nk, T* out,
              const ggms_opts* opts, void* stream) {
  if (n <= 0 || nk < 0) return GGMS_E_INVALID_ARG;
  ggms_opts o;
  if (read_opts(opts, &o) != GGMS_OK) return GGMS_E_INVALID_ARG;
  Context* c = (Context*)cx;
  if (!c) {
    int rc = default_context(&c);
    if (rc) return rc;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  return run_single_tuned<T>(c, d_in, (uint64_t)n, ks, (uint64_t)nk, out, o, (cudaStream_t)stream);
}


// ------------------------------------------------------------------ batched segmented path
// Every caller segment that holds a k: small ones are finished straight from
// the input (one warp or one CTA each); the others get sample-quantile bins at
// level 0, and the children of those bins go through radix levels (or
// straight to the warp / CTA finishers) -- every level runs over all segments
// at once.
template <typename T>
static int run_segmented(Context* ctx, const T* d_in, const int64_t* seg_off, int64_t nseg64,
                         const uint32_t* ks, const int64_t* k_off, T* out, const ggms_opts& o,
                         cudaStream_t st, int lv_mult = 8) {
  using K = typename KeyOf<T>::K;
  if (!d_in || !seg_off || !k_off || nseg64 <= 0 || nseg64 > (1 << 30)) return GGMS_E_INVALID_ARG;
  if ((uintptr_t)d_in % sizeof(T) != 0) return GGMS_E_INVALID_ARG;
  const uint32_t nseg = (uint32_t)nseg64;
  int64_t h_tot[2], h_k[2];
  GGMS_CU(cudaSetDevice(ctx->device));
  GGMS_CU(cudaMemcpyAsync(&h_tot[0], seg_off, 8, cudaMemcpyDeviceToHost, st));
  GGMS_CU(cudaMemcpyAsync(&h_tot[1], seg_off + nseg, 8, cudaMemcpyDeviceToHost, st));
  GGMS_CU(cudaMemcpyAsync(&h_k[0], k_off, 8, cudaMemcpyDeviceToHost, st));
  GGMS_CU(cudaMemcpyAsync(&h_k[1], k_off + nseg, 8, cudaMemcpyDeviceToHost, st));
  GGMS_CU(cudaStreamSynchronize(st));
  if (h_tot[0] != 0 || h_k[0] != 0 || h_tot[1] < 0 || h_k[1] < 0) return GGMS_E_INVALID_ARG;
  const uint64_t n = (uint64_t)h_tot[1];
  const uint64_t nk64 = (uint64_t)h_k[1];
  if (nk64 == 0) return GGMS_OK;
  if (n == 0 || n > 0xFFFFFFFFull || nk64 > 0x7FFFFFFFull || !ks || !out) return GGMS_E_INVALID_ARG;
  const uint32_t nk = (uint32_t)nk64;
  ggms_opts oo = o;
  oo.assigner = GGMS_ASSIGNER_SAMPLED;
  oo.num_buckets = 1024;
  oo.sample_size = 1024;
  Plan p;
  int rc = make_plan(&p, n, nk, oo);
  if (rc) return rc;
  const uint32_t small_keys = (uint32_t)(SMALL_SMEM / sizeof(K));
  p.cap_seg = std::max<uint32_t>(nk, nseg) + 1;
  p.cap_tiles = (uint32_t)((n + TILE - 1) / TILE) + p.cap_seg;
  p.cap_q = (uint32_t)std::min<uint64_t>(nseg, n / QSAMP) + 1;
  Workspace<K> w0 = layout<K>(p, sizeof(T), nullptr);
  rc = ensure_arena(ctx, w0.bytes);
  if (rc) return rc;
  Workspace<K> w = layout<K>(p, sizeof(T), ctx->arena);
  const Caps caps{p.cap_seg, p.cap_tiles, p.nk, small_keys, tiny_keys<K>()};
  // the stream-ordered part: captured once and replayed when the call repeats
  auto enqueue = [&](cudaStream_t s) -> int {
    GGMS_CU(cudaMemsetAsync(w.C, 0, sizeof(Counters), s));
    ++ctx->launches;
    seg_init<K><<<cdiv(nseg, 256), 256, 0, s>>>(seg_off, nseg, k_off, w.segs[0], w.tiles[0], w.khead[0],
                                                 w.smalls, w.tinies, w.bigs[0], p.cap_q, w.C, caps);
    ++ctx->launches;
    seg_set_count<<<1, 1, 0, s>>>(w.C, nseg);
    ++ctx->launches;
    k_init_seg<K><<<cdiv(nk, 256), 256, 0, s>>>(ks, nk, seg_off, k_off, nseg, w.segs[0], w.khead[0], w.knext,
                                                 w.krank, w.kseg, w.C);
    // small caller segments, straight from the input
    rc = launch_small_select<T>(ctx, d_in, w.segs[0], w.khead[0], w, caps, s, k_off);
    if (rc) return rc;
    ++ctx->launches;
    seg_sample<T><<<ctx->sms * 2, 1024, 0, s>>>(d_in, w.segs[0], w.bigs[0], w.C, p.cap_q, w.qtab, w.qdir,
                                                 p.seed ^ 0x5E6A11ull);
    // level 0 over the input with quantile bins; then radix levels over candidates
    // (a child range of up to 2^bits keys needs ceil(bits / 11) more levels)
    const int maxlev = 1 + (KeyBits<K>::value + RADIX_BITS - 1) / RADIX_BITS;
    const int lv_grid = ctx->sms * lv_mult;
    const int seg_grid = ctx->sms * 2;
    for (int l = 0; l < maxlev; ++l) {
      const int pp = l & 1, q = pp ^ 1;
      K* dst = w.cand[l & 1];
      const K* src = w.cand[(l + 1) & 1];  // the previous level's candidates (l >= 1)
      ++ctx->launches;
      lvl_prep<<<ctx->sms * 2, 256, 0, s>>>(w.rows[pp], w.aflag[pp], w.bigs[pp], w.C, pp, caps);
      ++ctx->launches;
      if (l == 0)
        lvl_count<T, LV_NT, true><<<lv_grid, LV_NT, 0, s>>>(d_in, w.segs[pp], w.tiles[pp], w.C, pp, w.rows[pp],
                                                             caps, w.qtab, w.qdir);
      else
        lvl_count<K, LV_NT><<<lv_grid, LV_NT, 0, s>>>(src, w.segs[pp], w.tiles[pp], w.C, pp, w.rows[pp], caps,
                                                       nullptr, nullptr);
      ++ctx->launches;
      lvl_scan<<<seg_grid, 1024, 0, s>>>(w.rows[pp], w.bigs[pp], w.C, pp, caps);
      ++ctx->launches;
      lvl_locate_rows<<<cdiv(nk, 256), 256, 0, s>>>(w.rows[pp], NBIN, nk, w.krank, w.kseg, w.kbin,
                                                       w.aflag[pp], NBIN_WORDS, w.C);
      ++ctx->launches;
      if (l == 0)
        lvl_children<K, 1024, true><<<seg_grid, 1024, 0, s>>>(w.rows[pp], w.aflag[pp], w.segs[pp], w.C, pp,
                                                               w.segs[q], w.cursor[q], w.tiles[q], w.points,
                                                               w.khead[q], w.smalls, w.tinies, w.bigs[pp],
                                                               w.bigs[q], caps, w.qtab);
      else
        lvl_children<K, 1024><<<seg_grid, 1024, 0, s>>>(w.rows[pp], w.aflag[pp], w.segs[pp], w.C, pp,
                                                         w.segs[q], w.cursor[q], w.tiles[q], w.points,
                                                         w.khead[q], w.smalls, w.tinies, w.bigs[pp],
                                                         w.bigs[q], caps, nullptr);
      ++ctx->launches;
      lvl_relabel<K><<<cdiv(nk, 256), 256, 0, s>>>(w.rows[pp], NBIN, nk, w.kbin, w.kseg, w.kkey,
                                                      w.points, w.C, w.segs[q], w.khead[q], w.knext);
      if (l + 1 < maxlev) {
        ++ctx->launches;
        if (l == 0)
          lvl_compact<T, LV_NT, true><<<lv_grid, LV_NT, 0, s>>>(d_in, w.segs[pp], w.tiles[pp], w.C, pp,
                                                                 w.rows[pp], w.segs[q], w.cursor[q], dst, caps,
                                                                 w.qtab, w.qdir);
        else
          lvl_compact<K, LV_NT><<<lv_grid, LV_NT, 0, s>>>(src, w.segs[pp], w.tiles[pp], w.C, pp,
                                                           w.rows[pp], w.segs[q], w.cursor[q], dst, caps,
                                                           nullptr, nullptr);
        rc = launch_small_select<K>(ctx, dst, w.segs[q], w.khead[q], w, caps, s);
        if (rc) return rc;
      }
    }
    ++ctx->launches;
    write_out<T><<<cdiv(nk, 256), 256, 0, s>>>(w.kkey, w.kseg, nk, out, w.C);
  return cudaGetLastError() == cudaSuccess ? GGMS_OK : GGMS_E_CUDA;
  };
  if (o.stats || ctx->profile) {
    rc = enqueue(st);
  } else {
    const uint64_t key[] = {0x5E6ull + sizeof(T), (uint64_t)(uintptr_t)d_in, (uint64_t)(uintptr_t)seg_off, nseg,
                            (uint64_t)(uintptr_t)ks, (uint64_t)(uintptr_t)k_off, (uint64_t)(uintptr_t)out, n,
                            nk, (uint64_t)(uintptr_t)ctx->arena, (uint64_t)std::is_signed<T>::value,
                            (uint64_t)std::is_floating_point<T>::value, (uint64_t)lv_mult};
    rc = run_graphed(ctx, key, (int)(sizeof(key) / sizeof(key[0])), st, enqueue);
  }
  if (rc) return rc;
  rc = mark_done(ctx, st);
  if (rc) return rc;
  if (o.stats) {
    Counters hc;
    GGMS_CU(cudaMemcpyAsync(&hc, w.C, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    GGMS_CU(cudaStreamSynchronize(st));
    memset(o.stats, 0, sizeof(ggms_stats));
    o.stats->levels = (int32_t)hc.levels_run;
    o.stats->refine_elements = (int64_t)hc.refine_elems;
    o.stats->full_passes = (int32_t)hc.passes;
    if (hc.status) return (int)hc.status;
  }
  return GGMS_OK;
}

template <typename T>
static int run_segmented_tuned(Context* c, const T* d_in, const int64_t* seg_off, int64_t nseg,
                               const uint32_t* ks, const int64_t* k_off, T* out, const ggms_opts& o,
                               cudaStream_t st) {
  if (!o.autotune || o.stats) return run_segmented<T>(c, d_in, seg_off, nseg, ks, k_off, out, o, st);
  // the class needs n and K: read the totals (run_segmented reads them again)
  int64_t h[2] = {0, 0};
  if (nseg <= 0 || !seg_off || !k_off) return GGMS_E_INVALID_ARG;
  GGMS_CU(cudaSetDevice(c->device));
  GGMS_CU(cudaMemcpyAsync(&h[0], seg_off + nseg, 8, cudaMemcpyDeviceToHost, st));
  GGMS_CU(cudaMemcpyAsync(&h[1], k_off + nseg, 8, cudaMemcpyDeviceToHost, st));
  GGMS_CU(cudaStreamSynchronize(st));
  const uint64_t key[4] = {0x5E60000ull | sizeof(T) | (std::is_floating_point<T>::value ? 32u : 0u),
                           (uint64_t)bitlen64((uint64_t)std::max<int64_t>(h[0], 0)) |
                               ((uint64_t)bitlen64((uint64_t)std::max<int64_t>(h[1], 0)) << 8) |
                               ((uint64_t)bitlen64((uint64_t)nseg) << 16),
                           0ull, 0ull};
  if (const Context::Tuned* t = tuned_find(c, key))
    return run_segmented<T>(c, d_in, seg_off, nseg, ks, k_off, out, o, st, t->lv_mult);
  static const int mults[] = {4, 8, 16};
  float best = 3.4e38f;
  Context::Tuned pick{{key[0], key[1], key[2], key[3]}, 0, 0, 0, 8};
  for (int m : mults) {
    float ms = 0.0f;
    const int rc = time_calls(st, [&] { return run_segmented<T>(c, d_in, seg_off, nseg, ks, k_off, out, o, st, m); },
                              &ms);
    if (rc) return rc;
    if (ms < best) {
      best = ms;
      pick.lv_mult = m;
    }
  }
  c->tuned.push_back(pick);
  return run_segmented<T>(c, d_in, seg_off, nseg, ks, k_off, out, o, st, pick.lv_mult);
}

template <typename T>
static int segmented(ggms_context* cx, const T* d_in, const int64_t* seg_off, int64_t nseg,
                     const uint32_t* ks, const int64_t* k_off, T* out, const ggms_opts* opts,
                     void* stream) {
  ggms_opts o;
  if (read_opts(opts, &o) != GGMS_OK) return GGMS_E_INVALID_ARG;
  Context* c = (Context*)cx;
  if (!c) {
    int rc = default_context(&c);
    if (rc) return rc;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  return run_segmented_tuned<T>(c, d_in, seg_off, nseg, ks, k_off, out, o, (cudaStream_t)stream);
}



GGMS_END
