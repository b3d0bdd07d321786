// sobol_tables.cpp -- direction-vector and scramble-constant getters of the C ABI
// (library/src/rocrand.cpp:590-634).  The tables arrive with the Sobol generators; until
// then every set is reported as unavailable (OUT_OF_RANGE, the reference's answer for an
// unknown set).
#include "common.hpp"

extern "C" {

rocrand_status ROCRANDAPI rocrand_get_direction_vectors32(const unsigned int**         vectors,
                                                          rocrand_direction_vector_set set)
{
    (void)vectors;
    (void)set;
    return ROCRAND_STATUS_OUT_OF_RANGE;
}

rocrand_status ROCRANDAPI rocrand_get_direction_vectors64(const unsigned long long**   vectors,
                                                          rocrand_direction_vector_set set)
{
    (void)vectors;
    (void)set;
    return ROCRAND_STATUS_OUT_OF_RANGE;
}

rocrand_status ROCRANDAPI rocrand_get_scramble_constants32(const unsigned int** constants)
{
    (void)constants;
    return ROCRAND_STATUS_OUT_OF_RANGE;
}

rocrand_status ROCRANDAPI rocrand_get_scramble_constants64(const unsigned long long** constants)
{
    (void)constants;
    return ROCRAND_STATUS_OUT_OF_RANGE;
}

} // extern "C"
