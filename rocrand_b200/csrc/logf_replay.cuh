// logf_replay.cuh -- the host C library's logf, reproduced on the device for the inputs of
// the inverse-erf normal.
//
// The reference's host generators compute the Sobol normal as
// sqrt(2) * erfinv(2p - 1) with erfinv(x) = sgn sqrt(-tt1 + sqrt(tt1^2 - tt2)), where tt1 and
// tt2 are linear in logf((1 - x)(1 + x)) (rocrand_normal.h:174-194, 228-233).  The outer
// difference cancels, so a logf result one ulp away moves the normal by tens of ulps: the
// normal can only match the host's if the logarithm is the host's, bit for bit.  The host's
// logf (glibc) is not correctly rounded: on the ~11.6 million distinct arguments this
// formula can produce, 0.93 % of its results are the other neighbour of the exact value.
//
// Method.  The device evaluates a logarithm L to about one double ulp (precise_math.cuh
// log_unit) and rounds it to float, f.  The host's result differs from f only where the
// exact value lies close to the midpoint between f and its neighbour on the side of L.  The
// build (rocrand_b200/data/make_logf_replay.cpp) runs the host's logf over every argument
// the formula can reach and records
//  * per bucket of arguments (the float's bits >> kBucketShift), the largest distance from
//    the midpoint, in units of 2^-16 ulp (plus one), of an argument where the host's result
//    differs from f (0: none in the bucket);
//  * the differing arguments with the host's result, in an open-addressing hash table.
// An argument whose distance is within its bucket's bound looks itself up (a few percent of
// arguments); all others return f.  The build then replays every reachable argument through
// this same code on the host and requires the host's logf result for each.  f is IEEE
// operations only and the distance and lookup integer ones, so the host and device builds
// of this header agree bit for bit.
#pragma once

#include "precise_math.cuh"

#include <cstdint>
#include <cstring>

namespace rb200
{
namespace lr
{

constexpr int      kBucketShift = 17;
constexpr uint32_t kBuckets     = (0x3f800000u >> kBucketShift) + 1; // arguments in (0, 1]
constexpr uint32_t kHashMul     = 0x9E3779B1u;                       // Fibonacci hashing

// The tables as the kernels see them (device pointers).
struct Table
{
    const uint16_t* bound = nullptr; // kBuckets entries
    const uint32_t* slots = nullptr; // (argument bits, result bits) pairs; argument 0 = empty
    uint32_t        log2_slots = 0;
    uint32_t        max_probe  = 0; // longest probe sequence of any stored argument
};

RB_PM_HD uint32_t fbits(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    return u;
}

RB_PM_HD float ffrom(uint32_t u)
{
    float x;
    memcpy(&x, &u, 4);
    return x;
}

// The device's own float logarithm f of t, and the distance of its double value L from the
// rounding boundary between the two floats around L, in units of 2^-16 float ulp (0 ..
// 32768; larger = safer).  L's double mantissa carries 29 bits below the float's last bit;
// they place L between the two floats (|L| > 2^-26 here, so L is a normal float number and
// both floats share its exponent or the larger one is the next power of two), and the
// boundary sits at 2^28 of them: integer operations only.
RB_PM_HD float base(float t, uint32_t& dist)
{
    const double   L   = pm::log_unit(static_cast<double>(t));
    const uint32_t low = static_cast<uint32_t>(pm::bits_of(L)) & 0x1fffffffu;
    const uint32_t off = low > (1u << 28) ? low - (1u << 28) : (1u << 28) - low;
    dist               = off >> 13;
    return static_cast<float>(L);
}

// The host C library's logf(t) for an argument of the inverse-erf normal.
RB_PM_HD float logf_host(float t, const Table& tb)
{
    if(!(t > 0.0f) || !(t <= 1.0f))
        return pm::logf(t); // zero (-inf) and anything outside the formula's range
    uint32_t    dist;
    const float f   = base(t, dist);
    const uint32_t key = fbits(t);
#if defined(__CUDA_ARCH__)
    const uint32_t bound = __ldg(tb.bound + (key >> kBucketShift));
#else
    const uint32_t bound = tb.bound[key >> kBucketShift];
#endif
    if(bound == 0u || dist > bound)
        return f;
    const uint32_t mask = (1u << tb.log2_slots) - 1u;
    uint32_t       h    = (key * kHashMul) >> (32 - tb.log2_slots);
    for(uint32_t k = 0; k < tb.max_probe; k++, h = (h + 1u) & mask)
    {
#if defined(__CUDA_ARCH__)
        const uint2    s  = __ldg(reinterpret_cast<const uint2*>(tb.slots) + h);
        const uint32_t sk = s.x, sv = s.y;
#else
        const uint32_t sk = tb.slots[2 * h], sv = tb.slots[2 * h + 1];
#endif
        if(sk == key)
            return ffrom(sv);
        if(sk == 0u)
            break;
    }
    return f;
}

} // namespace lr
} // namespace rb200
