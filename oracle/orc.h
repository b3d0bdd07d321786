/*
 * orc.h -- CPU oracle for rocRAND's host-API generation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * *host* generators (rocrand_create_generator_host_blocking) used as the parity
 * checker for the CUDA library.  Only tests/, __graft_entry__.smoke() and the
 * bench's cpu_baseline / reference legs may load it, and only as a checker or a
 * timed CPU baseline, never as a product path.
 *
 * Every entry point mirrors one reference C-ABI function (library/src/rocrand.cpp)
 * with the same argument meaning and the same rocrand_status codes, so a test can
 * drive the oracle and the CUDA library with the same call sequence.
 */
#ifndef ORC_H_
#define ORC_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_gen orc_gen;

int orc_create(orc_gen** g, int rng_type);
int orc_destroy(orc_gen* g);
int orc_initialize(orc_gen* g);
int orc_set_seed(orc_gen* g, unsigned long long seed);
int orc_set_seed_uint4(orc_gen* g, uint32_t x, uint32_t y, uint32_t z, uint32_t w);
int orc_set_offset(orc_gen* g, unsigned long long offset);
int orc_set_ordering(orc_gen* g, int order);
int orc_set_dimensions(orc_gen* g, unsigned int dims);

int orc_generate(orc_gen* g, uint32_t* out, size_t n);
int orc_generate_long_long(orc_gen* g, uint64_t* out, size_t n);
int orc_generate_char(orc_gen* g, uint8_t* out, size_t n);
int orc_generate_short(orc_gen* g, uint16_t* out, size_t n);
int orc_generate_uniform(orc_gen* g, float* out, size_t n);
int orc_generate_uniform_double(orc_gen* g, double* out, size_t n);
int orc_generate_uniform_half(orc_gen* g, uint16_t* out, size_t n);
int orc_generate_normal(orc_gen* g, float* out, size_t n, float mean, float stddev);
int orc_generate_normal_double(orc_gen* g, double* out, size_t n, double mean, double stddev);
int orc_generate_normal_half(orc_gen* g, uint16_t* out, size_t n, uint16_t mean, uint16_t stddev);
int orc_generate_log_normal(orc_gen* g, float* out, size_t n, float mean, float stddev);
int orc_generate_log_normal_double(orc_gen* g, double* out, size_t n, double mean, double stddev);
int orc_generate_log_normal_half(orc_gen* g, uint16_t* out, size_t n, uint16_t mean, uint16_t stddev);
int orc_generate_poisson(orc_gen* g, uint32_t* out, size_t n, double lambda);

/* Helpers exposed for unit tests of the oracle itself. */
uint16_t orc_float_to_half(float f);
float    orc_half_to_float(uint16_t h);
/* Poisson table as the reference builds it (poisson.hpp calculate_poisson_probabilities,
 * discrete.hpp normalize + create_alias_table).  Returns size; prob/alias need >= capacity. */
unsigned orc_poisson_table(double lambda, double* prob, uint32_t* alias, unsigned* offset);
unsigned orc_poisson_capacity(double lambda);
/* Moves the host library's log and sin/cos results of the fp64 normal transforms by the
 * given numbers of ulps (test hook, see orc_internal.h; 0, 0 restores). */
void orc_set_libm_ulps(int log_ulps, int trig_ulps);

#ifdef __cplusplus
}
#endif
#endif
