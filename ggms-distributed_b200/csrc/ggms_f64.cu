// ggms_f64.cu -- the double instantiation of the selector: its drop-in,
// extended, top-k entry points (include/ggms.h).
#define GGMS_TU tu_f64
#include "ggms_engine.cuh"

using namespace ggms;

extern "C" {

int ggms_bucket_multiselect_f64(const double* d_vector, int length, const uint32_t* kVals, int numKs,
                                double* outputs, int blocks, int threads) {
  (void)blocks;  // the reference's launch hints; the library picks its own shapes
  (void)threads;
  return dropin<double>(d_vector, length, kVals, numKs, outputs);
}

int ggms_iterative_smos_f64(const double* d_vector, int length, const uint32_t* kVals, int numKs,
                            double* outputs, int blocks, int threads) {
  (void)blocks;
  (void)threads;
  return dropin<double>(d_vector, length, kVals, numKs, outputs);
}

int ggms_multiselect_f64_ex(ggms_context* ctx, const double* d_in, int64_t n, const uint32_t* ks, int64_t nk,
                            double* out, const ggms_opts* opts, void* stream) {
  return ex<double>(ctx, d_in, n, ks, nk, out, opts, stream);
}

int ggms_topk_f64(ggms_context* ctx, const double* d_in, int64_t n, int64_t K, double* out, const ggms_opts* opts,
                  void* stream) {
  return topk_call<double>(ctx, d_in, n, K, out, opts, stream);
}

}  // extern "C"
