// ggms_mlp.cuh -- monotone 1-32-32-1 MLP CDF model (trained on the GPU).
#pragma once
#include "ggms_learned.cuh"

namespace ggms {

template <typename K>
static int mlp_fit_and_compile(const K* sorted, uint32_t S, int steps_opt, Assigner<K>* As,
                               LearnState* L, cudaStream_t st, long long* launches) {
  (void)launches;
  (void)sorted; (void)S; (void)steps_opt; (void)As; (void)L; (void)st;
  return GGMS_E_UNSUPPORTED;
}

}  // namespace ggms
