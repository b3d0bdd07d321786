// launch.cuh -- launch sizing and vector stores shared by the generator kernels.
#pragma once

#include "common.hpp"

#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

namespace rb200
{

constexpr unsigned kBlock = 256;

// 16-byte streaming store: outputs are written once and never re-read by the kernel,
// so they are marked evict-first to keep L2 for the engine state and tables.
__device__ __forceinline__ void store16_cs(void* p, uint4 v)
{
    __stcs(reinterpret_cast<uint4*>(p), v);
}

// Packs ow*opt values of T (16 bytes) into a uint4.
template<class T, unsigned N>
__host__ __device__ __forceinline__ uint4 pack16(const T (&v)[N])
{
    static_assert(sizeof(T) * N == 16, "16-byte vectors only");
    uint4 r;
    memcpy(&r, v, 16);
    return r;
}

// Resident blocks per SM of kernel `fn` with `smem` bytes of dynamic shared memory on the
// current device, computed once per (device, kernel, smem) and cached: a one-entry cache per
// thread in front of a shared table (two instantiations can share a kernel type, and a
// Poisson kernel's shared memory grows with its table, so the key holds both).
inline int blocks_per_sm(const void* fn, size_t smem)
{
    const int                  dev      = device_info().device;
    thread_local const void*   last_fn  = nullptr;
    thread_local size_t        last_smem = 0;
    thread_local int           last_dev = -1;
    thread_local int           last_per = 1;
    if(fn == last_fn && smem == last_smem && dev == last_dev)
        return last_per;
    static std::mutex                                               mu;
    static std::map<std::tuple<int, const void*, size_t>, int>      cache;
    int                                                             per = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        const auto                  it = cache.find(std::make_tuple(dev, fn, smem));
        if(it != cache.end())
            per = it->second;
    }
    if(per == 0)
    {
        if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kBlock, smem) != cudaSuccess || per < 1)
        {
            cudaGetLastError();
            per = 1;
        }
        std::lock_guard<std::mutex> lock(mu);
        cache[std::make_tuple(dev, fn, smem)] = per;
    }
    last_fn   = fn;
    last_smem = smem;
    last_dev  = dev;
    last_per  = per;
    return per;
}

// Grid for a grid-stride kernel over `work` items: enough resident blocks to fill every
// SM, never more than the work needs.
template<class Kernel>
inline unsigned grid_for(Kernel k, unsigned long long work, size_t smem)
{
    const int                per  = blocks_per_sm(reinterpret_cast<const void*>(k), smem);
    const unsigned long long full = static_cast<unsigned long long>(device_info().sm_count)
                                    * static_cast<unsigned long long>(per);
    const unsigned long long need = (work + kBlock - 1) / kBlock;
    unsigned long long       g    = need < full ? need : full;
    return static_cast<unsigned>(g < 1 ? 1 : g);
}

inline rocrand_status launch_status()
{
    return cudaGetLastError() == cudaSuccess ? ROCRAND_STATUS_SUCCESS
                                             : ROCRAND_STATUS_LAUNCH_FAILURE;
}

} // namespace rb200
