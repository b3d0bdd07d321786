// noalloc.cu -- Poisson generation that allocates nothing.
//
// Some callers cannot allocate device memory at all: code running inside a CUDA graph
// capture or a driver callback, allocators that forbid cudaMalloc after start-up, or
// processes whose memory is fully pre-partitioned.  rocrand_generate_poisson needs a
// scratch table (the alias table of lambda) in device memory, which a generator allocates
// on first use.  rocrand_b200_generate_poisson_noalloc produces the same values as a fresh
// Philox4x32-10 generator (seed, offset) calling rocrand_generate_poisson, but keeps its
// table in the file-scope array below, so neither it nor anything it calls allocates:
//  * the array holds up to kNoallocTableEntries entries (4096, 48 KiB); every GPU that
//    loads the library holds it until the process exits;
//  * a table larger than that is rejected with ROCRAND_STATUS_OUT_OF_RANGE (Poisson
//    tables for lambda <= 4000 have at most 2086 entries; larger lambdas need no table);
//  * the device address of the array is looked up once per device, by the first call
//    made on that device; make that first call before any stream capture;
//  * all calls share the array and each call rewrites the entries it uses, so calls that
//    overlap on the GPU (different streams, no ordering between them) race.
#include "common.hpp"
#include "generators.hpp"
#include "poisson.hpp"

#include <rocrand_b200.h>

#include <cmath>
#include <cstring>
#include <mutex>

namespace rb200
{

constexpr uint32_t kNoallocTableEntries = 4096;

// packed alias entries (poisson.hpp alias_entry); the alias array stays for the layout
static __device__ __align__(256) unsigned long long g_noalloc_thr[kNoallocTableEntries];
static __device__ __align__(256) uint32_t g_noalloc_alias[kNoallocTableEntries];

namespace
{

struct NoallocScratch
{
    unsigned long long* thr = nullptr;
    uint32_t* alias = nullptr;
};

// Device addresses of the arrays, looked up once per device with that device current.
rocrand_status scratch_for_current_device(NoallocScratch& out)
{
    static std::mutex     mu;
    static NoallocScratch cache[64];
    int                   dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    std::lock_guard<std::mutex> lock(mu);
    if(cache[dev].thr == nullptr)
    {
        void* p = nullptr;
        void* a = nullptr;
        if(cudaGetSymbolAddress(&p, g_noalloc_thr) != cudaSuccess
           || cudaGetSymbolAddress(&a, g_noalloc_alias) != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        cache[dev].thr   = static_cast<unsigned long long*>(p);
        cache[dev].alias = static_cast<uint32_t*>(a);
    }
    out = cache[dev];
    return ROCRAND_STATUS_SUCCESS;
}

// Host staging of one table, per calling thread (static storage: no heap allocation).
struct HostTable
{
    double   p[kNoallocTableEntries];
    double   prob[kNoallocTableEntries];
    unsigned long long thr[kNoallocTableEntries];
    uint32_t alias[kNoallocTableEntries];
    uint32_t small[kNoallocTableEntries];
    uint32_t large[kNoallocTableEntries];
};
thread_local HostTable t_table;

// The Poisson alias table of lambda built exactly as the generator path builds it
// (poisson.cpp, after library/src/rng/distribution/poisson.hpp:110-161 and
// discrete.hpp:189-265), on fixed-size arrays.  Returns false when it does not fit.
bool build_table(double lambda, uint32_t& size, uint32_t& offset)
{
    const size_t capacity = 2 * static_cast<size_t>(16.0 * (2.0 + std::sqrt(lambda)));
    if(capacity > kNoallocTableEntries)
        return false;
    HostTable&   t          = t_table;
    const double p_epsilon  = 1e-12;
    const double log_lambda = std::log(lambda);
    const int    left       = static_cast<int>(std::floor(lambda)) - static_cast<int>(capacity / 2);
    std::memset(t.p, 0, sizeof(double) * capacity);
    int lo = 0;
    for(int i = static_cast<int>(capacity / 2); i >= 0; i--)
    {
        const double x  = left + i;
        const double pp = std::exp(x * log_lambda - std::lgamma(x + 1.0) - lambda);
        if(pp < p_epsilon)
        {
            lo = i + 1;
            break;
        }
        t.p[i] = pp;
    }
    int hi = static_cast<int>(capacity) - 1;
    for(int i = static_cast<int>(capacity / 2) + 1; i < static_cast<int>(capacity); i++)
    {
        const double x  = left + i;
        const double pp = std::exp(x * log_lambda - std::lgamma(x + 1.0) - lambda);
        if(pp < p_epsilon)
        {
            hi = i - 1;
            break;
        }
        t.p[i] = pp;
    }
    for(int i = lo; i <= hi; i++)
        t.p[i - lo] = t.p[i];
    size   = static_cast<uint32_t>(hi - lo + 1);
    offset = static_cast<uint32_t>(left + lo);
    double sum = 0.0;
    for(uint32_t i = 0; i < size; i++)
        sum += t.p[i];
    for(uint32_t i = 0; i < size; i++)
        t.p[i] /= sum;

    const double average = 1.0 / size;
    uint32_t     ns = 0, nl = 0;
    for(uint32_t i = 0; i < size; i++)
    {
        t.prob[i]  = 0.0;
        t.alias[i] = 0;
        if(t.p[i] >= average)
            t.large[nl++] = i;
        else
            t.small[ns++] = i;
    }
    while(ns > 0 && nl > 0)
    {
        const uint32_t less = t.small[--ns];
        const uint32_t more = t.large[--nl];
        t.prob[less]        = t.p[less] * size;
        t.alias[less]       = more;
        t.p[more]           = (t.p[more] + t.p[less]) - average;
        if(t.p[more] >= average)
            t.large[nl++] = more;
        else
            t.small[ns++] = more;
    }
    for(uint32_t i = 0; i < ns; i++)
        t.prob[t.small[i]] = 1.0;
    for(uint32_t i = 0; i < nl; i++)
        t.prob[t.large[i]] = 1.0;
    for(uint32_t i = 0; i < size; i++)
        t.thr[i] = alias_entry(t.prob[i], t.alias[i]);
    return true;
}

} // namespace

} // namespace rb200

using namespace rb200;

extern "C" rocrand_status ROCRANDAPI
    rocrand_b200_generate_poisson_noalloc(unsigned long long seed,
                                          unsigned long long offset,
                                          unsigned int*      output_data,
                                          size_t             n,
                                          double             lambda,
                                          cudaStream_t       stream)
{
    if(lambda <= 0.0)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        DistParams p;
        if(lambda > kPoissonHugeLambda)
        {
            p.huge        = 1;
            p.lambda      = lambda;
            p.sqrt_lambda = std::sqrt(lambda);
            return philox_poisson_with_table(seed, offset, output_data, n, p, stream);
        }
        NoallocScratch s;
        rocrand_status st = scratch_for_current_device(s);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        uint32_t size = 0, table_offset = 0;
        if(!build_table(lambda, size, table_offset))
            return ROCRAND_STATUS_OUT_OF_RANGE;
        if(output_data == nullptr || n == 0)
            return ROCRAND_STATUS_SUCCESS;
        // Pageable sources: each copy returns once the source has been read, so the
        // per-thread staging can be reused by the next call.
        if(cudaMemcpyAsync(s.thr, t_table.thr, sizeof(unsigned long long) * size, cudaMemcpyHostToDevice, stream)
               != cudaSuccess
           || cudaMemcpyAsync(s.alias, t_table.alias, sizeof(uint32_t) * size,
                              cudaMemcpyHostToDevice, stream)
                  != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        p.huge   = 0;
        p.thr    = s.thr;
        p.alias  = s.alias;
        p.size   = size;
        p.offset = table_offset;
        p.lambda = lambda;
        return philox_poisson_with_table(seed, offset, output_data, n, p, stream);
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}
