/*
 * Names-only HIP -> CUDA shim used to compile the reference's own sources (read in
 * place, never copied) into oracle/_ref.  TEST INFRASTRUCTURE ONLY.
 *
 * Two flavours:
 *  - default (REF_CPU_ONLY defined): every runtime call the reference's *host*
 *    generators make is answered on the CPU (malloc/memcpy/inline host funcs), so the
 *    host generators run in a container without a GPU;
 *  - REF_CPU_ONLY undefined: the calls forward to the CUDA runtime, so the reference's
 *    device generators can run on a GPU.
 * Only the HIP names the reference uses are provided (library/src/**, library/include/**).
 */
#ifndef REFSHIM_HIP_RUNTIME_H_
#define REFSHIM_HIP_RUNTIME_H_

#ifndef __HIP_PLATFORM_NVCC__
    #define __HIP_PLATFORM_NVCC__ 1
#endif
#ifndef __HIP_PLATFORM_NVIDIA__
    #define __HIP_PLATFORM_NVIDIA__ 1
#endif
#if defined(__CUDA_ARCH__) && !defined(__HIP_DEVICE_COMPILE__)
    #define __HIP_DEVICE_COMPILE__ 1
#endif

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdint.h>
#include <cstring>

typedef cudaError_t  hipError_t;
typedef cudaStream_t hipStream_t;
typedef cudaHostFn_t hipHostFn_t;
typedef cudaMemcpyKind hipMemcpyKind;
typedef cudaDeviceProp hipDeviceProp_t;

#define hipSuccess cudaSuccess
#define hipErrorUnknown cudaErrorUnknown
#define hipErrorInvalidHandle cudaErrorInvalidResourceHandle
#define hipErrorOutOfMemory cudaErrorMemoryAllocation
#define hipMemcpyHostToDevice cudaMemcpyHostToDevice
#define hipMemcpyDeviceToHost cudaMemcpyDeviceToHost
#define hipMemcpyDeviceToDevice cudaMemcpyDeviceToDevice
#define hipMemcpyHostToHost cudaMemcpyHostToHost
#define hipMemcpyDefault cudaMemcpyDefault
#define hipStreamNonBlocking cudaStreamNonBlocking
#define hipStreamPerThread cudaStreamPerThread

/* Warp shuffles of the pre-sync form, full mask. */
#if defined(__CUDA_ARCH__)
    #define __shfl(...) __shfl_sync(0xffffffffu, __VA_ARGS__)
    #define __shfl_up(...) __shfl_up_sync(0xffffffffu, __VA_ARGS__)
    #define __shfl_down(...) __shfl_down_sync(0xffffffffu, __VA_ARGS__)
#endif

inline const char* hipGetErrorName(hipError_t e) { return cudaGetErrorName(e); }
inline hipError_t  hipGetDevice(int* d) { return cudaGetDevice(d); }
inline hipError_t  hipGetDeviceProperties(hipDeviceProp_t* p, int d)
{
    return cudaGetDeviceProperties(p, d);
}
inline int hipGetStreamDeviceId(hipStream_t) { return 0; }

#if defined(REF_CPU_ONLY)

inline hipError_t hipMalloc(void** p, size_t n)
{
    *p = std::malloc(n ? n : 1);
    return *p ? hipSuccess : hipErrorOutOfMemory;
}
template<class T>
inline hipError_t hipMalloc(T** p, size_t n)
{
    return hipMalloc(reinterpret_cast<void**>(p), n);
}
inline hipError_t hipFree(void* p)
{
    std::free(p);
    return hipSuccess;
}
inline hipError_t hipHostMalloc(void** p, size_t n)
{
    *p = std::malloc(n ? n : 1);
    return *p ? hipSuccess : hipErrorOutOfMemory;
}
template<class T>
inline hipError_t hipHostMalloc(T** p, size_t n)
{
    return hipHostMalloc(reinterpret_cast<void**>(p), n);
}
inline hipError_t hipHostFree(void* p)
{
    std::free(p);
    return hipSuccess;
}
inline hipError_t hipMemcpy(void* d, const void* s, size_t n, hipMemcpyKind)
{
    std::memcpy(d, s, n);
    return hipSuccess;
}
inline hipError_t hipMemcpyAsync(void* d, const void* s, size_t n, hipMemcpyKind, hipStream_t)
{
    std::memcpy(d, s, n);
    return hipSuccess;
}
inline hipError_t hipDeviceSynchronize() { return hipSuccess; }
inline hipError_t hipGetLastError() { return hipSuccess; }
inline hipError_t hipLaunchHostFunc(hipStream_t, hipHostFn_t fn, void* data)
{
    fn(data);
    return hipSuccess;
}
inline hipError_t hipStreamGetFlags(hipStream_t, unsigned int* f)
{
    *f = 0;
    return hipSuccess;
}

#else

template<class T>
inline hipError_t hipMalloc(T** p, size_t n)
{
    return cudaMalloc(reinterpret_cast<void**>(p), n);
}
inline hipError_t hipFree(void* p) { return cudaFree(p); }
template<class T>
inline hipError_t hipHostMalloc(T** p, size_t n)
{
    return cudaMallocHost(reinterpret_cast<void**>(p), n);
}
inline hipError_t hipHostFree(void* p) { return cudaFreeHost(p); }
inline hipError_t hipMemcpy(void* d, const void* s, size_t n, hipMemcpyKind k)
{
    return cudaMemcpy(d, s, n, k);
}
inline hipError_t hipMemcpyAsync(void* d, const void* s, size_t n, hipMemcpyKind k, hipStream_t st)
{
    return cudaMemcpyAsync(d, s, n, k, st);
}
inline hipError_t hipDeviceSynchronize() { return cudaDeviceSynchronize(); }
inline hipError_t hipGetLastError() { return cudaGetLastError(); }
inline hipError_t hipLaunchHostFunc(hipStream_t st, hipHostFn_t fn, void* data)
{
    return cudaLaunchHostFunc(st, fn, data);
}
inline hipError_t hipStreamGetFlags(hipStream_t st, unsigned int* f)
{
    return cudaStreamGetFlags(st, f);
}

#endif

#endif
