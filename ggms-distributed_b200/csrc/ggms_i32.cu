// ggms_i32.cu -- the int32_t instantiation of the selector: its drop-in,
// extended, top-k entry points (include/ggms.h).
#define GGMS_TU tu_i32
#include "ggms_engine.cuh"

using namespace ggms;

extern "C" {

int ggms_bucket_multiselect_i32(const int32_t* d_vector, int length, const uint32_t* kVals, int numKs,
                                int32_t* outputs, int blocks, int threads) {
  (void)blocks;  // the reference's launch hints; the library picks its own shapes
  (void)threads;
  return dropin<int32_t>(d_vector, length, kVals, numKs, outputs);
}

int ggms_iterative_smos_i32(const int32_t* d_vector, int length, const uint32_t* kVals, int numKs,
                            int32_t* outputs, int blocks, int threads) {
  (void)blocks;
  (void)threads;
  return dropin<int32_t>(d_vector, length, kVals, numKs, outputs);
}

int ggms_multiselect_i32_ex(ggms_context* ctx, const int32_t* d_in, int64_t n, const uint32_t* ks, int64_t nk,
                            int32_t* out, const ggms_opts* opts, void* stream) {
  return ex<int32_t>(ctx, d_in, n, ks, nk, out, opts, stream);
}

int ggms_topk_i32(ggms_context* ctx, const int32_t* d_in, int64_t n, int64_t K, int32_t* out, const ggms_opts* opts,
                  void* stream) {
  return topk_call<int32_t>(ctx, d_in, n, K, out, opts, stream);
}

}  // extern "C"
