// common.hpp -- shared host-side definitions of librocrand (B200 build).
//
// The generator object replaces the reference's type-erased vtable
// (library/src/rng/generator_type.hpp:28-291): one C++ class per generator family, all
// deriving from the opaque rocrand_generator_base_type of the C ABI.
#pragma once

#include <rocrand/rocrand.h>

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace rb200
{

// Distribution requested by one generate call.  One value per reference entry point
// (rocrand.cpp:212-377); the generator maps it onto its own functor family.
enum class Dist : int
{
    U32 = 0,
    U8,
    U16,
    U64,
    F32,
    F64,
    F16,
    NORMAL_F32,
    NORMAL_F64,
    NORMAL_F16,
    LOGNORMAL_F32,
    LOGNORMAL_F64,
    LOGNORMAL_F16,
    POISSON
};

// Parameters of a distribution, passed by value into kernels.
struct DistParams
{
    float    mean_f = 0.f, std_f = 1.f;
    double   mean_d = 0.0, std_d = 1.0;
    uint16_t mean_h = 0, std_h = 0x3c00;
    // Poisson: alias table (device pointers) or the normal approximation above 4000.
    const double*   prob        = nullptr;
    const unsigned long long* thr = nullptr; // packed alias entries (poisson.hpp alias_entry)
    const uint32_t* alias       = nullptr;
    const double*   cdf         = nullptr;
    uint32_t        size        = 0;
    uint32_t        offset      = 0;
    double          lambda      = 0.0;
    double          sqrt_lambda = 0.0;
    int             huge        = 0;
};

// Bytes of one output element of each distribution.
inline size_t dist_elem_size(Dist d)
{
    switch(d)
    {
        case Dist::U8: return 1;
        case Dist::U16:
        case Dist::F16:
        case Dist::NORMAL_F16:
        case Dist::LOGNORMAL_F16: return 2;
        case Dist::U64:
        case Dist::F64:
        case Dist::NORMAL_F64:
        case Dist::LOGNORMAL_F64: return 8;
        default: return 4;
    }
}

// Reference stride contracts (config/config_defaults.hpp:33-108 via the NVIDIA default
// configs): the output order of a few corner cases depends on these grid sizes, so the
// kernels reproduce them arithmetically whatever grid they actually launch.
constexpr uint32_t kPhiloxRefStride   = 1024u * 256u; // Philox / ThreeFry grid
constexpr uint32_t kStatefulEngines   = 512u * 256u;  // XORWOW / MRG / LFSR113 engines

// Device properties needed for launch sizing, cached per device.
struct DeviceInfo
{
    int device   = 0;
    int sm_count = 148;
};
const DeviceInfo& device_info();

struct BatchReq; // batch.hpp

} // namespace rb200

// Base of every generator: the opaque handle type of the C ABI.
struct rocrand_generator_base_type
{
    virtual ~rocrand_generator_base_type() = default;

    virtual rocrand_rng_type type() const = 0;
    virtual rocrand_status   init()       = 0;

    virtual rocrand_status set_seed(unsigned long long seed) = 0;
    virtual rocrand_status set_seed_uint4(uint4 seed)
    {
        (void)seed;
        return ROCRAND_STATUS_TYPE_ERROR;
    }
    virtual rocrand_status set_offset(unsigned long long offset) = 0;
    virtual rocrand_status set_order(rocrand_ordering order)     = 0;
    virtual rocrand_status set_dimensions(unsigned int dims)
    {
        (void)dims;
        return ROCRAND_STATUS_TYPE_ERROR;
    }
    virtual rocrand_status set_stream(cudaStream_t stream)
    {
        m_stream = stream;
        return ROCRAND_STATUS_SUCCESS;
    }
    // Positions the generator at output `index` of the stream that a fresh generator of the
    // same type and seed (offset 0) writes with distribution d in one call, so that the next
    // call of d continues that stream from there (rocrand_b200_set_output_position).
    virtual rocrand_status set_output_position(rb200::Dist d, unsigned long long index)
    {
        (void)d, (void)index;
        return ROCRAND_STATUS_TYPE_ERROR;
    }
    // One generate call: data is device memory of n elements of the distribution's type.
    virtual rocrand_status generate(void* data, size_t n, rb200::Dist d, const rb200::DistParams& p)
        = 0;
    virtual rocrand_status generate_poisson(unsigned int* data, size_t n, double lambda) = 0;
    // Batched-fill form of the next call: describes `n` values of batch distribution `dist`
    // (batch.hpp) into `data` as a descriptor of the batch kernel, from the generator's
    // current state, and advances the state exactly as that call would.  Poisson tables are
    // made resident on `stream`.  TYPE_ERROR where the generator has no batched form.
    virtual rocrand_status batch_descriptor(uint32_t dist, double p0, double p1, void* data,
                                            size_t n, rb200::BatchReq& r, cudaStream_t stream)
    {
        (void)dist, (void)p0, (void)p1, (void)data, (void)n, (void)r, (void)stream;
        return ROCRAND_STATUS_TYPE_ERROR;
    }

    cudaStream_t stream() const { return m_stream; }

    // Host execution: generate calls write host memory, computed on the CPU by the same
    // engine and distribution code as the kernels (host generators of a process with no GPU,
    // host_generator.cpp).  Families without a CPU form return false.
    virtual bool set_host_execution() { return false; }
    bool         host_execution() const { return m_host_exec; }

protected:
    cudaStream_t m_stream    = 0;
    bool         m_host_exec = false;
};
