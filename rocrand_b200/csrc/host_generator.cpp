// host_generator.cpp -- rocrand_create_generator_host / _host_blocking.
//
// The reference's host generators write into host memory with the same values as its
// device generators (library/src/rng/generator_type.hpp:128-177, rocrand.cpp:111-160), and
// run on the CPU (system.hpp:140-214).  Here a host generator takes one of two forms:
//  * in a process with no CUDA device (or with ROCRAND_B200_HOST_CPU=1 in the environment),
//    the generator itself in host execution: every generate call runs on the CPU, through
//    the same engine, output-order and distribution code as the kernels (compiled for the
//    host; fp32 transcendentals from the C library, as the reference's host path takes
//    them), spread over the host's cores;
//  * otherwise the device generator of the same type, whose outputs are copied into the
//    caller's host buffer: each generate call runs the device kernel into a scratch buffer
//    that has the same address modulo 256 bytes as the host buffer (the output layout --
//    head, aligned vectors, tail -- depends on the address), then copies the n values out
//    on the generator's stream and waits for them.  So the non-blocking flavour returns
//    with its outputs complete as the blocking one does, which its contract allows.
#include "common.hpp"
#include "generators.hpp"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <memory>

namespace rb200
{
namespace
{

class HostGenerator final : public rocrand_generator_base_type
{
public:
    explicit HostGenerator(rocrand_generator_base_type* inner) : m_inner(inner) {}
    ~HostGenerator() override { cudaFree(m_scratch); }

    rocrand_rng_type type() const override { return m_inner->type(); }
    rocrand_status   init() override { return m_inner->init(); }
    rocrand_status   set_seed(unsigned long long seed) override { return m_inner->set_seed(seed); }
    rocrand_status   set_seed_uint4(uint4 seed) override { return m_inner->set_seed_uint4(seed); }
    rocrand_status   set_offset(unsigned long long offset) override { return m_inner->set_offset(offset); }
    rocrand_status   set_order(rocrand_ordering order) override { return m_inner->set_order(order); }
    rocrand_status   set_dimensions(unsigned int dims) override { return m_inner->set_dimensions(dims); }
    rocrand_status   set_stream(cudaStream_t stream) override
    {
        m_stream = stream;
        return m_inner->set_stream(stream);
    }

    rocrand_status generate(void* data, size_t n, Dist d, const DistParams& p) override
    {
        if(data == nullptr || n == 0)
            return m_inner->generate(data, n, d, p);
        void*          dev = nullptr;
        rocrand_status st  = stage(data, n, dist_elem_size(d), dev);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        st = m_inner->generate(dev, n, d, p);
        return st == ROCRAND_STATUS_SUCCESS ? copy_out(data, dev, n * dist_elem_size(d)) : st;
    }

    rocrand_status generate_poisson(unsigned int* data, size_t n, double lambda) override
    {
        if(data == nullptr || n == 0)
            return m_inner->generate_poisson(data, n, lambda);
        void*          dev = nullptr;
        rocrand_status st  = stage(data, n, sizeof(unsigned int), dev);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        st = m_inner->generate_poisson(static_cast<unsigned int*>(dev), n, lambda);
        return st == ROCRAND_STATUS_SUCCESS ? copy_out(data, dev, n * sizeof(unsigned int)) : st;
    }

private:
    // A device address congruent to `host` modulo 256 with n elements of `elem` bytes behind
    // it (a count whose byte size would wrap cannot be a real host buffer: refused).
    rocrand_status stage(const void* host, size_t n, size_t elem, void*& dev)
    {
        if(n > (SIZE_MAX - 256) / elem)
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        const size_t need = n * elem + 256;
        if(need > m_cap)
        {
            // the previous scratch may still be read by work queued on the stream
            if(m_scratch != nullptr && cudaStreamSynchronize(m_inner->stream()) != cudaSuccess)
                return ROCRAND_STATUS_INTERNAL_ERROR;
            cudaFree(m_scratch);
            m_scratch = nullptr;
            m_cap     = 0;
            if(cudaMalloc(&m_scratch, need) != cudaSuccess)
            {
                m_scratch = nullptr;
                return ROCRAND_STATUS_ALLOCATION_FAILED;
            }
            m_cap = need;
        }
        dev = static_cast<unsigned char*>(m_scratch) + reinterpret_cast<uintptr_t>(host) % 256;
        return ROCRAND_STATUS_SUCCESS;
    }

    rocrand_status copy_out(void* host, const void* dev, size_t bytes)
    {
        const cudaStream_t s = m_inner->stream();
        if(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess
           || cudaStreamSynchronize(s) != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        return ROCRAND_STATUS_SUCCESS;
    }

    std::unique_ptr<rocrand_generator_base_type> m_inner;
    void*                                        m_scratch = nullptr;
    size_t                                       m_cap     = 0;
};

} // namespace

// No usable CUDA device, or host execution asked for.
static bool host_cpu_mode()
{
    const char* e = std::getenv("ROCRAND_B200_HOST_CPU");
    if(e != nullptr && e[0] != '\0' && e[0] != '0')
        return true;
    int count = 0;
    if(cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        return true;
    }
    return false;
}

rocrand_generator_base_type* make_host_generator(rocrand_rng_type t)
{
    rocrand_generator_base_type* inner = make_generator(t);
    if(inner == nullptr)
        return nullptr;
    if(host_cpu_mode() && inner->set_host_execution())
        return inner;
    return new HostGenerator(inner);
}

} // namespace rb200
