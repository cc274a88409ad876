/* ggms_generate.h -- device-side problem generators.
 *
 * The reference generates every test vector with cuRAND on the device and copies it
 * to the host before timing (DistributedSMOS/generateProblems.cu:43-513, tables at
 * :75-79, 438-446, 509-513).  These entry points fill a caller-owned device buffer
 * directly, so inputs of 2^30 elements and more need no host generation or upload.
 * `kind` is the index into the reference's generator table of that value type; the
 * values come from a counter-based hash of (seed, index), so a result depends only
 * on (kind, n, seed), not on the launch shape.  Not the cuRAND stream: the same seed
 * gives other numbers than the reference, with the same distribution.
 *
 * float kinds (namesOfFloatGeneratingFunctions):
 *   0 UNIFORM FLOATS      [0, 1), 24-bit grid
 *   1 NORMAL FLOATS       N(0, 1), Box-Muller
 *   2 KILLER FLOATS       kind 0's draw masked with 0x80EFFFFF (subnormals and the
 *                         lowest normal binade), sorted; then 2^-126 .. 2^126 in
 *                         the first min(n, 253) slots
 *   3 HALF NORMAL FLOATS  |N(0, 1)|
 *   4 NORMAL FLOATS 100   N(0, 100^2)
 *   5 HUGE UNIFORM FLOATS [0, 1) x 10^6
 *   6 NOISY FLOATS        floor(n/5) ones and the rest zeros, plus N(0, 0.01^2)
 *   7 ALL ONES FLOATS     1.0
 *   8 ONES TWOS FLOAT     floor(n/2) twos and the rest ones
 *   9 CAUCHY FLOAT        tan(pi (u - 1/2)), u in (0, 1)
 * double kinds: 0 UNIFORM DOUBLES [0, 1) (53-bit grid), 1 NORMAL DOUBLES N(0, 1),
 *   2 KILLER DOUBLES (kind 0's draw masked with 0x800FFFFFFFFFFFFF: subnormals,
 *   sorted; then 2^-1022 .. 2^1022 in the first min(n, 2045) slots).
 * uint32 kinds: 0 UNIFORM UNSIGNED INTEGERS, 1 SORTED UINTS (ascending: element i is
 *   drawn from the i-th of n equal strata of [0, 2^32), so the vector is sorted
 *   without a sort), 2 UNIFORM 0-4 (the reference's table entry writes i % 100).
 *
 * The two-valued float kinds (6, 8) place their values through the bijection
 * i -> (a i + b) mod n (a coprime to n, both drawn from the seed), so the counts
 * are exact and the positions scattered.  Those two and SORTED UINTS need
 * n <= 2^32.
 *
 * Returns GGMS_OK, GGMS_E_INVALID_ARG (null buffer, n <= 0, kind outside the table),
 * GGMS_E_UNSUPPORTED (n > 2^32 for float kinds 6, 8 and uint32 kind 1; n >= 2^31
 * for the KILLER kinds) or GGMS_E_CUDA.
 * Enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream); no host
 * synchronization.  No allocation, except that the KILLER kinds sort their draw
 * with CUB's device radix sort in stream-ordered scratch (cudaMallocAsync, freed
 * with cudaFreeAsync on the same stream; n elements plus CUB's temporaries).
 */
#ifndef GGMS_GENERATE_H
#define GGMS_GENERATE_H

#include <stdint.h>

#include "ggms.h"

#ifdef __cplusplus
extern "C" {
#endif

/* generateUniformFloats ... generateCauchyFloats (DistributedSMOS/generateProblems.cu:86-446),
 * generateBucketKillerFloats (:422-436) */
GGMS_API int ggms_generate_f32(float* d_out, int64_t n, int kind, uint64_t seed, void* stream);
/* generateUniformDoubles, generateNormalDoubles, generateBucketKillerDoubles
 * (DistributedSMOS/generateProblems.cu:456-513) */
GGMS_API int ggms_generate_f64(double* d_out, int64_t n, int kind, uint64_t seed, void* stream);
/* generateUniformUnsignedIntegers, generateSortedArrayUints, generateUniformZeroToFourUints
 * (DistributedSMOS/generateProblems.cu:43-79) */
GGMS_API int ggms_generate_u32(uint32_t* d_out, int64_t n, int kind, uint64_t seed, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GGMS_GENERATE_H */
