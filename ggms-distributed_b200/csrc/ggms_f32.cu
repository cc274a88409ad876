// ggms_f32.cu -- the float instantiation of the selector: its drop-in,
// extended, top-k and batched entry points (include/ggms.h).
#define GGMS_TU tu_f32
#include "ggms_engine.cuh"

using namespace ggms;

extern "C" {

int ggms_bucket_multiselect_f32(const float* d_vector, int length, const uint32_t* kVals, int numKs,
                                float* outputs, int blocks, int threads) {
  (void)blocks;  // the reference's launch hints; the library picks its own shapes
  (void)threads;
  return dropin<float>(d_vector, length, kVals, numKs, outputs);
}

int ggms_iterative_smos_f32(const float* d_vector, int length, const uint32_t* kVals, int numKs,
                            float* outputs, int blocks, int threads) {
  (void)blocks;
  (void)threads;
  return dropin<float>(d_vector, length, kVals, numKs, outputs);
}

int ggms_multiselect_f32_ex(ggms_context* ctx, const float* d_in, int64_t n, const uint32_t* ks, int64_t nk,
                            float* out, const ggms_opts* opts, void* stream) {
  return ex<float>(ctx, d_in, n, ks, nk, out, opts, stream);
}

int ggms_topk_f32(ggms_context* ctx, const float* d_in, int64_t n, int64_t K, float* out, const ggms_opts* opts,
                  void* stream) {
  return topk_call<float>(ctx, d_in, n, K, out, opts, stream);
}

int ggms_multiselect_segmented_f32(ggms_context* ctx, const float* d_in, const int64_t* seg_off, int64_t nseg,
                                   const uint32_t* ks, const int64_t* k_off, float* out, const ggms_opts* opts,
                                   void* stream) {
  return segmented<float>(ctx, d_in, seg_off, nseg, ks, k_off, out, opts, stream);
}

#ifdef GGMS_SETUP_TRACE
GGMS_API int ggms_trace_read_f32(unsigned long long* out) {
  return cudaMemcpyFromSymbol(out, ggms_trace_buf, sizeof(ggms_trace_buf)) == cudaSuccess ? 0 : 4;
}
GGMS_API int ggms_trace_read_cta_f32(unsigned long long* out) {
  return cudaMemcpyFromSymbol(out, ggms_trace_cta, sizeof(ggms_trace_cta)) == cudaSuccess ? 0 : 4;
}
#endif

}  // extern "C"
