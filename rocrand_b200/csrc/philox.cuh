// philox.cuh -- the Philox4x32-10 output contract as device helpers: call parameters,
// the value at a stream position, the sequential head/tail run and the 16-byte vector of
// one block.  Shared by the per-generator kernels (philox.cu) and the batched fill
// (batch.cu).
#pragma once

#include "common.hpp"
#include "counter_engines.cuh"
#include "dist.cuh"
#include "launch.cuh"

namespace rb200
{

struct PhiloxCall
{
    PhiloxKeys         keys;
    uint4              c0;     // engine counter at the call's first value
    uint32_t           s0;     // engine sub-position (0..3)
    uint32_t           head;   // elements before the first 16-byte boundary
    uint32_t           start0; // stream offset of vector 0 (thread 0 after the head)
    uint32_t           tail;   // elements after the last full vector
    unsigned char*     data;   // output base
    unsigned char*     vec;    // first 16-byte aligned output byte
    unsigned long long n;
    unsigned long long vec_n;
};

// Value at relative stream position p (sequential head/tail path only).
__host__ __device__ __forceinline__ uint32_t philox_value(const PhiloxCall& a, unsigned long long p)
{
    const unsigned long long q = a.s0 + p;
    const uint4              b = philox_block(ctr_add(a.c0, q >> 2), a.keys);
    return word_of(b, static_cast<uint32_t>(q & 3));
}

// Applies F sequentially from stream position `pos` and writes `count` elements at `out`
// (the reference's scalar head/tail loops, one engine() per input).
template<class F>
__host__ __device__ void philox_scalar_run(const PhiloxCall& a, const F& f, unsigned long long pos,
                                  typename F::T* out, uint32_t count)
{
    typename F::T v[F::ow];
    uint32_t      in[F::iw];
    for(uint32_t done = 0; done < count; done += F::ow)
    {
        for(unsigned i = 0; i < F::iw; i++)
            in[i] = philox_value(a, pos++);
        f(in, v);
        for(unsigned o = 0; o < F::ow && done + o < count; o++)
            out[done + o] = v[o];
    }
}

template<class F>
__host__ __device__ __forceinline__ uint4 philox_vec(const F& f, uint4 w)
{
    constexpr unsigned opt = 4 / F::iw;
    typename F::T      out[opt * F::ow];
    const uint32_t     in[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for(unsigned s = 0; s < opt; s++)
        f(in + s * F::iw, out + s * F::ow);
    return pack16(out);
}

} // namespace rb200
