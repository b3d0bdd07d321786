/*
 * rocrand.h -- drop-in host C ABI of the B200 random-number library (librocrand.so).
 *
 * Every type, enum value and function below keeps the name, signature and meaning of
 * the reference's library/include/rocrand/rocrand.h (rocRAND 3.2.0) so that code written
 * against rocRAND -- including its Python ctypes binding (python/rocrand/rocrand/rocrand.py)
 * and its C++ wrapper (rocrand.hpp) -- links against this library unchanged.  The stream
 * type is hipStream_t in the reference; on this CUDA build it is cudaStream_t.
 * Each declaration cites the reference declaration (rocrand.h) and implementation
 * (library/src/rocrand.cpp) it replaces.
 */
#ifndef ROCRAND_H_
#define ROCRAND_H_

#include <stddef.h>

#include <cuda_runtime_api.h>
#include <vector_types.h>

#if defined(__cplusplus)
    #include <cuda_fp16.h>
#endif

#include "rocrand/rocrand_discrete_types.h"

#ifndef ROCRANDAPI
    #define ROCRANDAPI __attribute__((visibility("default")))
#endif

/* Library version, 3.2.0 encoded as major*100000 + minor*100 + patch (rocrand_version.h.in). */
#define ROCRAND_VERSION 300200

/* Opaque generator handle (rocrand.h:41). */
typedef struct rocrand_generator_base_type* rocrand_generator;

/* half is the CUDA __half (rocrand.h:46); C callers get a bit-compatible 16-bit struct. */
#if defined(__cplusplus)
typedef __half half;
#else
typedef struct
{
    unsigned short x;
} half;
#endif

/* Stream type of the reference's API (hipStream_t) on CUDA. */
#ifndef ROCRAND_B200_HIP_STREAM_DEFINED
    #define ROCRAND_B200_HIP_STREAM_DEFINED
typedef cudaStream_t hipStream_t;
#endif

#define ROCRAND_DEFAULT_MAX_BLOCK_SIZE 256

#if defined(__cplusplus)
extern "C" {
#endif

/* Status codes (rocrand.h:59-71). */
typedef enum rocrand_status
{
    ROCRAND_STATUS_SUCCESS                   = 0,
    ROCRAND_STATUS_VERSION_MISMATCH          = 100,
    ROCRAND_STATUS_NOT_CREATED               = 101,
    ROCRAND_STATUS_ALLOCATION_FAILED         = 102,
    ROCRAND_STATUS_TYPE_ERROR                = 103,
    ROCRAND_STATUS_OUT_OF_RANGE              = 104,
    ROCRAND_STATUS_LENGTH_NOT_MULTIPLE       = 105,
    ROCRAND_STATUS_DOUBLE_PRECISION_REQUIRED = 106,
    ROCRAND_STATUS_LAUNCH_FAILURE            = 107,
    ROCRAND_STATUS_INTERNAL_ERROR            = 108
} rocrand_status;

/* Generator types (rocrand.h:77-99). */
typedef enum rocrand_rng_type
{
    ROCRAND_RNG_PSEUDO_DEFAULT          = 400,
    ROCRAND_RNG_PSEUDO_XORWOW           = 401,
    ROCRAND_RNG_PSEUDO_MRG32K3A         = 402,
    ROCRAND_RNG_PSEUDO_MTGP32           = 403,
    ROCRAND_RNG_PSEUDO_PHILOX4_32_10    = 404,
    ROCRAND_RNG_PSEUDO_MRG31K3P         = 405,
    ROCRAND_RNG_PSEUDO_LFSR113          = 406,
    ROCRAND_RNG_PSEUDO_MT19937          = 407,
    ROCRAND_RNG_PSEUDO_THREEFRY2_32_20  = 408,
    ROCRAND_RNG_PSEUDO_THREEFRY2_64_20  = 409,
    ROCRAND_RNG_PSEUDO_THREEFRY4_32_20  = 410,
    ROCRAND_RNG_PSEUDO_THREEFRY4_64_20  = 411,
    ROCRAND_RNG_QUASI_DEFAULT           = 500,
    ROCRAND_RNG_QUASI_SOBOL32           = 501,
    ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL32 = 502,
    ROCRAND_RNG_QUASI_SOBOL64           = 504,
    ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL64 = 505
} rocrand_rng_type;

/* Orderings (rocrand.h:106-114). */
typedef enum rocrand_ordering
{
    ROCRAND_ORDERING_PSEUDO_BEST    = 100,
    ROCRAND_ORDERING_PSEUDO_DEFAULT = 101,
    ROCRAND_ORDERING_PSEUDO_SEEDED  = 102,
    ROCRAND_ORDERING_PSEUDO_LEGACY  = 103,
    ROCRAND_ORDERING_PSEUDO_DYNAMIC = 104,
    ROCRAND_ORDERING_QUASI_DEFAULT  = 201
} rocrand_ordering;

/* Direction vector sets (rocrand.h:120-126). */
typedef enum rocrand_direction_vector_set
{
    ROCRAND_DIRECTION_VECTORS_32_JOEKUO6           = 101,
    ROCRAND_SCRAMBLED_DIRECTION_VECTORS_32_JOEKUO6 = 102,
    ROCRAND_DIRECTION_VECTORS_64_JOEKUO6           = 103,
    ROCRAND_SCRAMBLED_DIRECTION_VECTORS_64_JOEKUO6 = 104
} rocrand_direction_vector_set;

/* Lifecycle (rocrand.h:163-209; rocrand.cpp:115-210). */
rocrand_status ROCRANDAPI rocrand_create_generator(rocrand_generator* generator,
                                                   rocrand_rng_type   rng_type);
rocrand_status ROCRANDAPI rocrand_create_generator_host(rocrand_generator* generator,
                                                        rocrand_rng_type   rng_type);
rocrand_status ROCRANDAPI rocrand_create_generator_host_blocking(rocrand_generator* generator,
                                                                 rocrand_rng_type   rng_type);
rocrand_status ROCRANDAPI rocrand_destroy_generator(rocrand_generator generator);

/* Generation (rocrand.h:231-544; rocrand.cpp:212-377). */
rocrand_status ROCRANDAPI rocrand_generate(rocrand_generator generator,
                                           unsigned int*     output_data,
                                           size_t            n);
rocrand_status ROCRANDAPI rocrand_generate_long_long(rocrand_generator       generator,
                                                     unsigned long long int* output_data,
                                                     size_t                  n);
rocrand_status ROCRANDAPI rocrand_generate_char(rocrand_generator generator,
                                                unsigned char*    output_data,
                                                size_t            n);
rocrand_status ROCRANDAPI rocrand_generate_short(rocrand_generator generator,
                                                 unsigned short*   output_data,
                                                 size_t            n);
rocrand_status ROCRANDAPI rocrand_generate_uniform(rocrand_generator generator,
                                                   float*            output_data,
                                                   size_t            n);
rocrand_status ROCRANDAPI rocrand_generate_uniform_double(rocrand_generator generator,
                                                          double*           output_data,
                                                          size_t            n);
rocrand_status ROCRANDAPI rocrand_generate_uniform_half(rocrand_generator generator,
                                                        half*             output_data,
                                                        size_t            n);
rocrand_status ROCRANDAPI rocrand_generate_normal(
    rocrand_generator generator, float* output_data, size_t n, float mean, float stddev);
rocrand_status ROCRANDAPI rocrand_generate_normal_double(
    rocrand_generator generator, double* output_data, size_t n, double mean, double stddev);
rocrand_status ROCRANDAPI rocrand_generate_normal_half(
    rocrand_generator generator, half* output_data, size_t n, half mean, half stddev);
rocrand_status ROCRANDAPI rocrand_generate_log_normal(
    rocrand_generator generator, float* output_data, size_t n, float mean, float stddev);
rocrand_status ROCRANDAPI rocrand_generate_log_normal_double(
    rocrand_generator generator, double* output_data, size_t n, double mean, double stddev);
rocrand_status ROCRANDAPI rocrand_generate_log_normal_half(
    rocrand_generator generator, half* output_data, size_t n, half mean, half stddev);
rocrand_status ROCRANDAPI rocrand_generate_poisson(rocrand_generator generator,
                                                   unsigned int*     output_data,
                                                   size_t            n,
                                                   double            lambda);

/* Setters (rocrand.h:565-710; rocrand.cpp:379-449). */
rocrand_status ROCRANDAPI rocrand_initialize_generator(rocrand_generator generator);
rocrand_status ROCRANDAPI rocrand_set_stream(rocrand_generator generator, hipStream_t stream);
rocrand_status ROCRANDAPI rocrand_set_seed(rocrand_generator generator, unsigned long long seed);
rocrand_status ROCRANDAPI rocrand_set_seed_uint4(rocrand_generator generator, uint4 seed);
rocrand_status ROCRANDAPI rocrand_set_offset(rocrand_generator generator,
                                             unsigned long long offset);
rocrand_status ROCRANDAPI rocrand_set_ordering(rocrand_generator generator,
                                               rocrand_ordering  order);
rocrand_status ROCRANDAPI rocrand_set_quasi_random_generator_dimensions(rocrand_generator generator,
                                                                        unsigned int dimensions);

/* Misc (rocrand.h:723-829; rocrand.cpp:451-634). */
rocrand_status ROCRANDAPI rocrand_get_version(int* version);
rocrand_status ROCRANDAPI rocrand_create_poisson_distribution(
    double lambda, rocrand_discrete_distribution* discrete_distribution);
rocrand_status ROCRANDAPI
    rocrand_create_discrete_distribution(const double*                  probabilities,
                                         unsigned int                   size,
                                         unsigned int                   offset,
                                         rocrand_discrete_distribution* discrete_distribution);
rocrand_status ROCRANDAPI
    rocrand_destroy_discrete_distribution(rocrand_discrete_distribution discrete_distribution);
rocrand_status ROCRANDAPI rocrand_get_direction_vectors32(const unsigned int**         vectors,
                                                          rocrand_direction_vector_set set);
rocrand_status ROCRANDAPI rocrand_get_direction_vectors64(const unsigned long long**   vectors,
                                                          rocrand_direction_vector_set set);
rocrand_status ROCRANDAPI rocrand_get_scramble_constants32(const unsigned int** constants);
rocrand_status ROCRANDAPI rocrand_get_scramble_constants64(const unsigned long long** constants);

#if defined(__cplusplus)
}
#endif

#endif /* ROCRAND_H_ */
