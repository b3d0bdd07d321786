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
//    made on that device (whatever its lambda); make that first call before any stream
//    capture;
//  * each call writes its table into the array in stream order, through the parameters of
//    a small kernel (no host memory has to outlive the call);
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

// Host staging of one table, per calling thread: fixed-size arrays, so building a table
// allocates nothing on the device and no heap memory.  (A thread's first call may make the
// C library set up this thread-local block, as for any thread_local in a loaded library.)
struct HostTable
{
    double   p[kNoallocTableEntries];
    double   prob[kNoallocTableEntries];
    uint32_t alias[kNoallocTableEntries];
    uint32_t small[kNoallocTableEntries];
    uint32_t large[kNoallocTableEntries];
};
thread_local HostTable t_table;

// The Poisson alias table of lambda, built by the generator path's own builder (poisson.cpp,
// after library/src/rng/distribution/poisson.hpp:110-161 and discrete.hpp:189-265) on the
// fixed-size arrays above.  Returns false when it does not fit.
bool build_table(double lambda, uint32_t& size, uint32_t& offset)
{
    if(poisson_capacity(lambda) > kNoallocTableEntries)
        return false;
    HostTable& t = t_table;
    poisson_probabilities_into(lambda, t.p, size, offset);
    build_alias_into(t.p, size, t.prob, t.alias, t.small, t.large);
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
    if(!(lambda > 0.0)) // also refuses NaN
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        // Every call, whatever its lambda, first makes sure this device's scratch address
        // is known, so that the first call on a device is the one that looks it up.
        NoallocScratch s;
        rocrand_status st = scratch_for_current_device(s);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        DistParams p;
        if(lambda > kPoissonHugeLambda)
        {
            p.huge        = 1;
            p.lambda      = lambda;
            p.sqrt_lambda = std::sqrt(lambda);
            return philox_poisson_with_table(seed, offset, output_data, n, p, stream);
        }
        uint32_t size = 0, table_offset = 0;
        if(!build_table(lambda, size, table_offset) || size > kPoissonTableCap)
            return ROCRAND_STATUS_OUT_OF_RANGE;
        if(output_data == nullptr || n == 0)
            return ROCRAND_STATUS_SUCCESS;
        // The table travels as kernel parameters (stream-ordered; nothing on the host must
        // outlive the call), as the generators' own tables do.
        st = upload_alias_entries(s.thr, s.alias, t_table.prob, t_table.alias, size, stream);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
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
