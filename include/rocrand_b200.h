/*
 * rocrand_b200.h -- entry points of librocrand that extend the rocRAND C ABI.
 *
 * Everything in include/rocrand/rocrand.h keeps the reference's meaning; the functions
 * below are additions of this library.
 */
#ifndef ROCRAND_B200_H_
#define ROCRAND_B200_H_

#include "rocrand/rocrand.h"

#if defined(__cplusplus)
extern "C" {
#endif

/*
 * Poisson values that need no device allocation.  No counterpart in the reference.
 *
 * Writes the n values that a fresh ROCRAND_RNG_PSEUDO_PHILOX4_32_10 generator with this
 * seed and offset would write with rocrand_generate_poisson(output_data, n, lambda) on
 * `stream`, without allocating anything: for callers that cannot call cudaMalloc (inside a
 * CUDA graph capture or a driver callback, or with device memory fully pre-partitioned).
 * Its scratch (the alias table of lambda, up to 4096 entries) is a fixed 48 KiB array that
 * every GPU loading the library holds until the process exits; lambda <= 0 and tables
 * beyond 4096 entries give ROCRAND_STATUS_OUT_OF_RANGE.  The first call on a device looks
 * up the array's address and should come before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race.
 */
rocrand_status ROCRANDAPI rocrand_b200_generate_poisson_noalloc(unsigned long long seed,
                                                                unsigned long long offset,
                                                                unsigned int*      output_data,
                                                                size_t             n,
                                                                double             lambda,
                                                                hipStream_t        stream);

#if defined(__cplusplus)
}
#endif

#endif /* ROCRAND_B200_H_ */
