/* ggms_diag.h -- diagnostic entry points of the learned bucket assigners.
 *
 * No reference counterpart (the reference has no learned component).  They
 * expose the GPU forward/backward kernels of the two CDF models so that their
 * gradients can be checked against a CPU restatement; they allocate and free
 * their own device memory and synchronize.  Not for the hot path.
 */
#ifndef GGMS_DIAG_H
#define GGMS_DIAG_H
#include <stdint.h>

#include "ggms.h"

#ifdef __cplusplus
extern "C" {
#endif

/* PL-CDF model.  sorted_keys: S ascending uint32 keys (host).  The knots are
 * built exactly as the selector builds them (1024 quantile knots, equal knots
 * merged); theta: 1024 raw parameters (host).  Returns the loss, the gradient
 * w.r.t. theta (first M entries; grad holds 1024), the M+1 knots (knots holds
 * 1025) and M. */
GGMS_API int ggms_diag_pl_gradient(const uint32_t* sorted_keys, int S, const float* theta,
                                   float* loss, float* grad, uint32_t* knots, int* M);

/* MLP-CDF model on 1024 explicit training points (x in [0,1], targets t):
 * loss and gradient w.r.t. the 1153 raw parameters (layout V1[32], c1[32],
 * V2[32][32] row-major by output unit, c2[32], V3[32], c3), computed by the
 * same cluster kernel that trains the model. */
GGMS_API int ggms_diag_mlp_gradient(const float* x, const float* t, const float* params,
                                    float* loss, float* grad);

/* Trains a model on the sorted keys with the selector's own kernels and
 * reports its training loss before/after and the bucket imbalance (max/mean
 * over 256 bucket groups on the sample) of the compiled assigner, next to the
 * sampled-pivot assigner's.  kind: GGMS_ASSIGNER_LEARNED_PL or _MLP. */
GGMS_API int ggms_diag_fit(const uint32_t* sorted_keys, int S, int kind, int steps,
                           float* loss_before, float* loss_after, float* imbalance_model,
                           float* imbalance_sampled);

#ifdef __cplusplus
}
#endif
#endif
