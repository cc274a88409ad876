// ggms_u32.cu -- the uint32_t instantiation of the selector: its drop-in,
// extended, top-k and batched entry points (include/ggms.h).
#define GGMS_TU tu_u32
#include "ggms_engine.cuh"

using namespace ggms;

extern "C" {

int ggms_bucket_multiselect_u32(const uint32_t* d_vector, int length, const uint32_t* kVals, int numKs,
                                uint32_t* outputs, int blocks, int threads) {
  (void)blocks;  // the reference's launch hints; the library picks its own shapes
  (void)threads;
  return dropin<uint32_t>(d_vector, length, kVals, numKs, outputs);
}

int ggms_iterative_smos_u32(const uint32_t* d_vector, int length, const uint32_t* kVals, int numKs,
                            uint32_t* outputs, int blocks, int threads) {
  (void)blocks;
  (void)threads;
  return dropin<uint32_t>(d_vector, length, kVals, numKs, outputs);
}

int ggms_multiselect_u32_ex(ggms_context* ctx, const uint32_t* d_in, int64_t n, const uint32_t* ks, int64_t nk,
                            uint32_t* out, const ggms_opts* opts, void* stream) {
  return ex<uint32_t>(ctx, d_in, n, ks, nk, out, opts, stream);
}

int ggms_topk_u32(ggms_context* ctx, const uint32_t* d_in, int64_t n, int64_t K, uint32_t* out, const ggms_opts* opts,
                  void* stream) {
  return topk_call<uint32_t>(ctx, d_in, n, K, out, opts, stream);
}

int ggms_multiselect_segmented_u32(ggms_context* ctx, const uint32_t* d_in, const int64_t* seg_off, int64_t nseg,
                                   const uint32_t* ks, const int64_t* k_off, uint32_t* out, const ggms_opts* opts,
                                   void* stream) {
  return segmented<uint32_t>(ctx, d_in, seg_off, nseg, ks, k_off, out, opts, stream);
}

}  // extern "C"
