// launch.cuh -- launch sizing and vector stores shared by the generator kernels.
#pragma once

#include "common.hpp"

#include <cuda_runtime.h>

#include <atomic>
#include <cstring>

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

// Grid for a grid-stride kernel over `work` items: enough resident blocks to fill every
// SM (occupancy of this kernel, cached per instantiation), never more than the work needs.
template<class Kernel>
inline unsigned grid_for(Kernel k, unsigned long long work, size_t smem)
{
    // threads launching the kernel for the first time may both compute it: same value
    static std::atomic<int> blocks_per_sm{0};
    int                     per = blocks_per_sm.load(std::memory_order_relaxed);
    if(per == 0)
    {
        if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, kBlock, smem) != cudaSuccess
           || per < 1)
            per = 1;
        blocks_per_sm.store(per, std::memory_order_relaxed);
    }
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
