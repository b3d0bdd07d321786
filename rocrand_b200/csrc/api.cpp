// api.cpp -- the extern "C" rocRAND host ABI of librocrand (B200 build).
//
// Same entry points, argument meaning and status codes as the reference's
// library/src/rocrand.cpp:111-634: a NULL generator gives NOT_CREATED, lambda <= 0 gives
// OUT_OF_RANGE, unknown generator types give TYPE_ERROR, and no C++ exception crosses the
// ABI (rocrand.cpp:92-99).
#include "common.hpp"
#include "generators.hpp"

#include <rocrand_b200.h>

#include <cuda_fp16.h>

#include <new>

namespace rb200
{

const DeviceInfo& device_info()
{
    // One entry per device, filled on first use on that device.
    static thread_local DeviceInfo cache[64];
    static thread_local bool       valid[64] = {};
    int                            dev       = 0;
    cudaGetDevice(&dev);
    if(dev < 0 || dev >= 64)
        dev = 0;
    if(!valid[dev])
    {
        int sms = 0;
        if(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess
           || sms <= 0)
            sms = 148;
        cache[dev].device   = dev;
        cache[dev].sm_count = sms;
        valid[dev]          = true;
    }
    return cache[dev];
}

rocrand_generator_base_type* make_generator(rocrand_rng_type t)
{
    switch(t)
    {
        case ROCRAND_RNG_PSEUDO_PHILOX4_32_10: return new PhiloxGenerator();
        case ROCRAND_RNG_PSEUDO_THREEFRY2_32_20:
        case ROCRAND_RNG_PSEUDO_THREEFRY2_64_20:
        case ROCRAND_RNG_PSEUDO_THREEFRY4_32_20:
        case ROCRAND_RNG_PSEUDO_THREEFRY4_64_20: return make_threefry(t);
        case ROCRAND_RNG_PSEUDO_DEFAULT:
        case ROCRAND_RNG_PSEUDO_XORWOW:
        case ROCRAND_RNG_PSEUDO_MRG32K3A:
        case ROCRAND_RNG_PSEUDO_MRG31K3P:
        case ROCRAND_RNG_PSEUDO_LFSR113: return make_stateful(t);
        case ROCRAND_RNG_PSEUDO_MT19937: return make_mt19937();
        case ROCRAND_RNG_PSEUDO_MTGP32: return make_mtgp32();
        case ROCRAND_RNG_QUASI_DEFAULT:
        case ROCRAND_RNG_QUASI_SOBOL32:
        case ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL32:
        case ROCRAND_RNG_QUASI_SOBOL64:
        case ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL64: return make_sobol(t);
        default: return nullptr;
    }
}

template<class Fn>
static rocrand_status guarded(Fn&& fn)
{
    try
    {
        return fn();
    }
    catch(const std::bad_alloc&)
    {
        return ROCRAND_STATUS_ALLOCATION_FAILED;
    }
    catch(rocrand_status s)
    {
        return s;
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

static uint16_t half_bits(half h)
{
    return __half_as_ushort(h);
}

} // namespace rb200

using namespace rb200;

extern "C" {

rocrand_status ROCRANDAPI rocrand_create_generator(rocrand_generator* generator,
                                                   rocrand_rng_type   rng_type)
{
    if(generator == nullptr)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    return guarded([&] {
        rocrand_generator_base_type* g = make_generator(rng_type);
        if(g == nullptr)
            return ROCRAND_STATUS_TYPE_ERROR;
        *generator = g;
        return ROCRAND_STATUS_SUCCESS;
    });
}

// Host generators (rocrand.cpp:118-160): outputs in host memory, values of the device
// generator of the same type (host_generator.cpp).
rocrand_status ROCRANDAPI rocrand_create_generator_host(rocrand_generator* generator,
                                                        rocrand_rng_type   rng_type)
{
    if(generator == nullptr)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    return guarded([&] {
        rocrand_generator_base_type* g = make_host_generator(rng_type);
        if(g == nullptr)
            return ROCRAND_STATUS_TYPE_ERROR;
        *generator = g;
        return ROCRAND_STATUS_SUCCESS;
    });
}

rocrand_status ROCRANDAPI rocrand_create_generator_host_blocking(rocrand_generator* generator,
                                                                 rocrand_rng_type   rng_type)
{
    return rocrand_create_generator_host(generator, rng_type);
}

rocrand_status ROCRANDAPI rocrand_destroy_generator(rocrand_generator generator)
{
    return guarded([&] {
        delete generator;
        return ROCRAND_STATUS_SUCCESS;
    });
}

#define RB200_GEN(generator, body)                   \
    do                                               \
    {                                                \
        if((generator) == nullptr)                   \
            return ROCRAND_STATUS_NOT_CREATED;       \
        return guarded([&] { return (body); });      \
    }                                                \
    while(0)

rocrand_status ROCRANDAPI rocrand_generate(rocrand_generator generator,
                                           unsigned int*     output_data,
                                           size_t            n)
{
    RB200_GEN(generator, generator->generate(output_data, n, Dist::U32, DistParams{}));
}

rocrand_status ROCRANDAPI rocrand_generate_long_long(rocrand_generator       generator,
                                                     unsigned long long int* output_data,
                                                     size_t                  n)
{
    RB200_GEN(generator, generator->generate(output_data, n, Dist::U64, DistParams{}));
}

rocrand_status ROCRANDAPI rocrand_generate_char(rocrand_generator generator,
                                                unsigned char*    output_data,
                                                size_t            n)
{
    RB200_GEN(generator, generator->generate(output_data, n, Dist::U8, DistParams{}));
}

rocrand_status ROCRANDAPI rocrand_generate_short(rocrand_generator generator,
                                                 unsigned short*   output_data,
                                                 size_t            n)
{
    RB200_GEN(generator, generator->generate(output_data, n, Dist::U16, DistParams{}));
}

rocrand_status ROCRANDAPI rocrand_generate_uniform(rocrand_generator generator,
                                                   float*            output_data,
                                                   size_t            n)
{
    RB200_GEN(generator, generator->generate(output_data, n, Dist::F32, DistParams{}));
}

rocrand_status ROCRANDAPI rocrand_generate_uniform_double(rocrand_generator generator,
                                                          double*           output_data,
                                                          size_t            n)
{
    RB200_GEN(generator, generator->generate(output_data, n, Dist::F64, DistParams{}));
}

rocrand_status ROCRANDAPI rocrand_generate_uniform_half(rocrand_generator generator,
                                                        half*             output_data,
                                                        size_t            n)
{
    RB200_GEN(generator, generator->generate(output_data, n, Dist::F16, DistParams{}));
}

static DistParams params_f(float mean, float stddev)
{
    DistParams p;
    p.mean_f = mean;
    p.std_f  = stddev;
    return p;
}

static DistParams params_d(double mean, double stddev)
{
    DistParams p;
    p.mean_d = mean;
    p.std_d  = stddev;
    return p;
}

static DistParams params_h(half mean, half stddev)
{
    DistParams p;
    p.mean_h = half_bits(mean);
    p.std_h  = half_bits(stddev);
    return p;
}

rocrand_status ROCRANDAPI rocrand_generate_normal(
    rocrand_generator generator, float* output_data, size_t n, float mean, float stddev)
{
    RB200_GEN(generator,
              generator->generate(output_data, n, Dist::NORMAL_F32, params_f(mean, stddev)));
}

rocrand_status ROCRANDAPI rocrand_generate_normal_double(
    rocrand_generator generator, double* output_data, size_t n, double mean, double stddev)
{
    RB200_GEN(generator,
              generator->generate(output_data, n, Dist::NORMAL_F64, params_d(mean, stddev)));
}

rocrand_status ROCRANDAPI rocrand_generate_normal_half(
    rocrand_generator generator, half* output_data, size_t n, half mean, half stddev)
{
    RB200_GEN(generator,
              generator->generate(output_data, n, Dist::NORMAL_F16, params_h(mean, stddev)));
}

rocrand_status ROCRANDAPI rocrand_generate_log_normal(
    rocrand_generator generator, float* output_data, size_t n, float mean, float stddev)
{
    RB200_GEN(generator,
              generator->generate(output_data, n, Dist::LOGNORMAL_F32, params_f(mean, stddev)));
}

rocrand_status ROCRANDAPI rocrand_generate_log_normal_double(
    rocrand_generator generator, double* output_data, size_t n, double mean, double stddev)
{
    RB200_GEN(generator,
              generator->generate(output_data, n, Dist::LOGNORMAL_F64, params_d(mean, stddev)));
}

rocrand_status ROCRANDAPI rocrand_generate_log_normal_half(
    rocrand_generator generator, half* output_data, size_t n, half mean, half stddev)
{
    RB200_GEN(generator,
              generator->generate(output_data, n, Dist::LOGNORMAL_F16, params_h(mean, stddev)));
}

rocrand_status ROCRANDAPI rocrand_generate_poisson(rocrand_generator generator,
                                                   unsigned int*     output_data,
                                                   size_t            n,
                                                   double            lambda)
{
    if(generator == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    if(!(lambda > 0.0)) // lambda <= 0 (and NaN)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    return guarded([&] { return generator->generate_poisson(output_data, n, lambda); });
}

rocrand_status ROCRANDAPI rocrand_initialize_generator(rocrand_generator generator)
{
    RB200_GEN(generator, generator->init());
}

rocrand_status ROCRANDAPI rocrand_set_stream(rocrand_generator generator, hipStream_t stream)
{
    RB200_GEN(generator, generator->set_stream(stream));
}

rocrand_status ROCRANDAPI rocrand_set_seed(rocrand_generator generator, unsigned long long seed)
{
    RB200_GEN(generator, generator->set_seed(seed));
}

rocrand_status ROCRANDAPI rocrand_set_seed_uint4(rocrand_generator generator, uint4 seed)
{
    RB200_GEN(generator, generator->set_seed_uint4(seed));
}

rocrand_status ROCRANDAPI rocrand_set_offset(rocrand_generator generator, unsigned long long offset)
{
    RB200_GEN(generator, generator->set_offset(offset));
}

// Addition of this library (include/rocrand_b200.h): no counterpart in the reference.
rocrand_status ROCRANDAPI rocrand_b200_set_output_position(rocrand_generator   generator,
                                                           rocrand_b200_output output,
                                                           unsigned long long  index)
{
    if(generator == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    if(static_cast<int>(output) < 0 || static_cast<int>(output) > static_cast<int>(Dist::POISSON))
        return ROCRAND_STATUS_OUT_OF_RANGE;
    return guarded([&] { return generator->set_output_position(static_cast<Dist>(output), index); });
}

rocrand_status ROCRANDAPI rocrand_set_ordering(rocrand_generator generator, rocrand_ordering order)
{
    RB200_GEN(generator, generator->set_order(order));
}

rocrand_status ROCRANDAPI rocrand_set_quasi_random_generator_dimensions(rocrand_generator generator,
                                                                        unsigned int dimensions)
{
    RB200_GEN(generator, generator->set_dimensions(dimensions));
}

rocrand_status ROCRANDAPI rocrand_get_version(int* version)
{
    if(version == nullptr)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    *version = ROCRAND_VERSION;
    return ROCRAND_STATUS_SUCCESS;
}

} // extern "C"
