/* ggms_noalloc.h -- a multiselect entry point that allocates no memory.
 *
 * No counterpart in the reference (FrzNo1/GGMS-Distributed): its wrappers
 * (DistributedSMOS/bucketMultiselect.cu:583-606, 805-845) cudaMalloc and
 * cudaFree their buffers inside every call, and the other entry points of this
 * library draw on a context workspace that grows with cudaMalloc.
 *
 * Who needs it: callers that must not allocate device memory while they run.
 * cudaMalloc and cudaFree synchronize the whole device (they stall every other
 * stream of the process), and they fail once a caching allocator (PyTorch's,
 * for one) has reserved the free memory -- so a latency-critical loop, or a
 * process whose device memory is already handed to a pool, cannot call an entry
 * point that may allocate.  This one works out of a fixed scratch region that
 * is part of the library's device image: the CUDA driver reserves it when it
 * loads the library's kernels, once per device, and it is never freed or grown.
 *
 * Limits: num_ks <= GGMS_NOALLOC_MAX_KS (the scratch holds the per-k state and
 * one 256-bin histogram per distinct key prefix, for at most that many ks); a
 * larger num_ks is rejected with GGMS_E_UNSUPPORTED before anything is
 * launched -- use ggms_multiselect_f32_ex for those.  1 <= n <= 2^32 - 1.
 */
#ifndef GGMS_NOALLOC_H
#define GGMS_NOALLOC_H

#include <stdint.h>

#include "ggms.h"

#define GGMS_NOALLOC_MAX_KS 1024
/* Size of the scratch region: the histograms (GGMS_NOALLOC_MAX_KS x 256
 * counters) plus four arrays of GGMS_NOALLOC_MAX_KS words of per-k and
 * per-prefix state and a 256-byte control block: 1,065,216 bytes per device. */
#define GGMS_NOALLOC_SCRATCH_BYTES (4u * (256u * GGMS_NOALLOC_MAX_KS + 4u * GGMS_NOALLOC_MAX_KS) + 256u)

#ifdef __cplusplus
extern "C" {
#endif

/* Exact k-th largest values of a float vector in device memory, like
 * ggms_multiselect_f32_ex, with no allocation: radix selection by 8-bit digits
 * (four passes over d_in), all state in the library's fixed scratch region.
 *
 * d_in:   device memory, n floats, not modified.
 * ks:     HOST memory, num_ks entries, 1-based k-th largest (k in [1, n]).  The
 *         values travel to the device inside the first kernel's launch
 *         arguments, so the array may be reused as soon as the call returns.
 * d_out:  DEVICE memory, num_ks floats: d_out[i] is the ks[i]-th largest.
 * stream: a cudaStream_t, or NULL for the legacy default stream.  The call only
 *         enqueues work (nine kernel launches) and returns without a host sync.
 *
 * Status: GGMS_OK; GGMS_E_INVALID_ARG for a null or misaligned pointer, n
 * outside [1, 2^32 - 1], num_ks < 0 or a k outside [1, n]; GGMS_E_UNSUPPORTED
 * for num_ks > GGMS_NOALLOC_MAX_KS; GGMS_E_CUDA when set-up or a launch fails,
 * or when the CUDA runtime already holds an error from earlier work on this
 * thread (the call then launches nothing and leaves that error for its owner).
 * Every argument is checked on the host before any CUDA call.  num_ks == 0
 * returns GGMS_OK and launches nothing.
 *
 * Set-up: every call looks up the address of the current device's scratch
 * region with cudaGetSymbolAddress (after the first call on a device this is a
 * lookup that allocates nothing; the first one makes the driver load the
 * library's kernels on that device if it has not yet).  Make the first call on
 * a device before any stream capture begins.
 *
 * Zero state: nothing in the scratch region needs to be zero on entry.  The
 * call's first kernel writes the per-k state and clears the level-0 histogram;
 * each later level clears the histogram rows of the next pass before it runs.
 *
 * Concurrency: there is ONE scratch region per device.  Two calls on the same
 * device whose work overlaps in time -- on different streams, or from different
 * host threads without ordering between them -- race on it and return wrong
 * answers.  Order such calls (one stream, or events between streams).  Calls
 * on different devices are independent. */
GGMS_API int ggms_multiselect_noalloc_f32(const float* d_in, int64_t n, const uint32_t* ks,
                                          int32_t num_ks, float* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GGMS_NOALLOC_H */
