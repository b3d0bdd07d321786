// counter_engines.cuh -- counter-based engines (Philox4x32-10, ThreeFry) as pure
// functions of a 128/256-bit counter, plus the host-side position arithmetic.
//
// The reference models these as stateful engines walked by discard/next calls
// (rocrand_philox4x32_10.h:208-308, rocrand_threefry4_impl.h:178-317).  Here the stream
// is addressed directly: value p of the stream is word (p mod W) of block(counter0 + p / W),
// so any thread can produce any output vector in one block evaluation.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace rb200
{

// ---- Philox4x32-10 (Random123 constants, rocrand_philox4x32_10.h:60-63) ----
constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

// The ten round keys of a seed: key + r * (W0, W1), computed once on the host so each
// round xors with a kernel-parameter constant.
struct PhiloxKeys
{
    uint32_t k[10][2];
};

inline PhiloxKeys philox_keys(unsigned long long seed)
{
    PhiloxKeys pk;
    uint32_t   k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
    for(int r = 0; r < 10; r++)
    {
        pk.k[r][0] = k0;
        pk.k[r][1] = k1;
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    return pk;
}

// Ten Philox rounds of one 128-bit counter (Random123's S-box: two 32x32->64 products).
__host__ __device__ __forceinline__ uint4 philox_block(uint4 c, const PhiloxKeys& pk)
{
#pragma unroll
    for(int r = 0; r < 10; r++)
    {
        const uint64_t p0 = static_cast<uint64_t>(kPhiloxM0) * c.x;
        const uint64_t p1 = static_cast<uint64_t>(kPhiloxM1) * c.z;
        c = make_uint4(static_cast<uint32_t>(p1 >> 32) ^ c.y ^ pk.k[r][0],
                       static_cast<uint32_t>(p1),
                       static_cast<uint32_t>(p0 >> 32) ^ c.w ^ pk.k[r][1],
                       static_cast<uint32_t>(p0));
    }
    return c;
}

// Philox blocks of counters (x0 + i, y, z, w) with y, z, w fixed across a launch (no carry
// out of the low word): the multiplies of rounds 1 and 2 whose operands are the fixed
// words are evaluated once on the host, so a block costs 18 instead of 20 wide multiplies.
struct PhiloxLane
{
    uint32_t a;    // round 1 word 0: hi(M1*z) ^ y ^ k0[0]
    uint32_t b;    // round 1 word 1: lo(M1*z)
    uint32_t wk;   // w ^ k0[1]
    uint32_t hima; // hi(M0*a)
    uint32_t loma; // lo(M0*a)
};

inline PhiloxLane philox_lane(uint4 c, const PhiloxKeys& pk)
{
    PhiloxLane     l;
    const uint64_t p1 = static_cast<uint64_t>(kPhiloxM1) * c.z;
    l.a               = static_cast<uint32_t>(p1 >> 32) ^ c.y ^ pk.k[0][0];
    l.b               = static_cast<uint32_t>(p1);
    l.wk              = c.w ^ pk.k[0][1];
    const uint64_t pa = static_cast<uint64_t>(kPhiloxM0) * l.a;
    l.hima            = static_cast<uint32_t>(pa >> 32);
    l.loma            = static_cast<uint32_t>(pa);
    return l;
}

__device__ __forceinline__ uint4 philox_block_lane(uint32_t x, const PhiloxLane& l,
                                                   const PhiloxKeys& pk)
{
    // round 1: only M0 * x varies
    const uint64_t p0 = static_cast<uint64_t>(kPhiloxM0) * x;
    const uint32_t c2 = static_cast<uint32_t>(p0 >> 32) ^ l.wk;
    const uint32_t d2 = static_cast<uint32_t>(p0);
    // round 2: word 0 is the fixed `a`, so only M1 * c2 varies
    const uint64_t p1 = static_cast<uint64_t>(kPhiloxM1) * c2;
    uint4          c  = make_uint4(static_cast<uint32_t>(p1 >> 32) ^ l.b ^ pk.k[1][0],
                                   static_cast<uint32_t>(p1), l.hima ^ d2 ^ pk.k[1][1], l.loma);
#pragma unroll
    for(int r = 2; r < 10; r++)
    {
        const uint64_t q0 = static_cast<uint64_t>(kPhiloxM0) * c.x;
        const uint64_t q1 = static_cast<uint64_t>(kPhiloxM1) * c.z;
        c = make_uint4(static_cast<uint32_t>(q1 >> 32) ^ c.y ^ pk.k[r][0],
                       static_cast<uint32_t>(q1),
                       static_cast<uint32_t>(q0 >> 32) ^ c.w ^ pk.k[r][1],
                       static_cast<uint32_t>(q0));
    }
    return c;
}

// 128-bit counter + 64-bit addend, with carries (the engine's discard_state arithmetic).
__host__ __device__ __forceinline__ uint4 ctr_add(uint4 c, uint64_t a)
{
    const uint64_t lo  = (static_cast<uint64_t>(c.y) << 32 | c.x);
    const uint64_t nlo = lo + a;
    const uint64_t hi  = (static_cast<uint64_t>(c.w) << 32 | c.z) + (nlo < lo ? 1u : 0u);
    return make_uint4(static_cast<uint32_t>(nlo), static_cast<uint32_t>(nlo >> 32),
                      static_cast<uint32_t>(hi), static_cast<uint32_t>(hi >> 32));
}

// Position of a 4-word counter engine: value index = 4 * counter + sub (mod 2^130).
struct CounterPos
{
    uint4    counter = {0, 0, 0, 0};
    uint32_t sub     = 0;

    // Advances by k values (the engine's discard(k), rocrand_philox4x32_10.h:208-218).
    void advance(unsigned long long k)
    {
        const unsigned long long q = sub + (k & 3ull);
        counter                    = ctr_add(counter, (k >> 2) + (q >> 2));
        sub                        = static_cast<uint32_t>(q & 3ull);
    }
};

// Words s..s+3 of the 8-word concatenation (a, b): the engine's interleave.
__host__ __device__ __forceinline__ uint4 interleave4(uint4 a, uint4 b, uint32_t s)
{
    switch(s)
    {
        case 1: return make_uint4(a.y, a.z, a.w, b.x);
        case 2: return make_uint4(a.z, a.w, b.x, b.y);
        case 3: return make_uint4(a.w, b.x, b.y, b.z);
        default: return a;
    }
}

__host__ __device__ __forceinline__ uint32_t word_of(uint4 v, uint32_t i)
{
    switch(i)
    {
        case 0: return v.x;
        case 1: return v.y;
        case 2: return v.z;
        default: return v.w;
    }
}

} // namespace rb200
