// stateful_engines.cuh -- step functions of the XORWOW, MRG32k3a, MRG31k3p and LFSR113
// engines, their jump-table application and small vector stores; shared by the
// per-generator kernels (stateful.cu), the batched fill (batch.cu) and the CPU path of the
// host generators (stateful.cu), which runs the same functions compiled for the host.
#pragma once

#include "common.hpp"

#include <cstring>

namespace rb200
{

// Read-only load: through the non-coherent cache on the device, a plain load on the host.
template<class T>
__host__ __device__ __forceinline__ T ld_ro(const T* p)
{
#if defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}

// ---- engines (step functions; the state is NW 32-bit words) ----

struct XorwowEngine // rocrand_xorwow.h:165-177
{
    static constexpr int kWords  = 6; // x[0..4], d
    static constexpr int kGf2    = 5; // words covered by the jump matrices
    static constexpr int kUnroll = 5; // steps after which the state words are back in place
    uint32_t             w[kWords];
    __host__ __device__ __forceinline__ uint32_t next()
    {
        const uint32_t t = w[0] ^ (w[0] >> 2);
        w[0]             = w[1];
        w[1]             = w[2];
        w[2]             = w[3];
        w[3]             = w[4];
        w[4]             = (w[4] ^ (w[4] << 4)) ^ (t ^ (t << 1));
        w[5] += 362437u;
        return w[5] + w[4];
    }
};

struct Lfsr113Engine // rocrand_lfsr113.h:146-160
{
    static constexpr int kWords  = 4;
    static constexpr int kGf2    = 4;
    static constexpr int kUnroll = 4; // fill iterations unrolled together: consecutive transforms overlap
    uint32_t             w[kWords];
    __host__ __device__ __forceinline__ uint32_t next()
    {
        uint32_t b;
        b    = ((w[0] << 6) ^ w[0]) >> 13;
        w[0] = ((w[0] & 4294967294u) << 18) ^ b;
        b    = ((w[1] << 2) ^ w[1]) >> 27;
        w[1] = ((w[1] & 4294967288u) << 2) ^ b;
        b    = ((w[2] << 13) ^ w[2]) >> 21;
        w[2] = ((w[2] & 4294967280u) << 7) ^ b;
        b    = ((w[3] << 3) ^ w[3]) >> 12;
        w[3] = ((w[3] & 4294967168u) << 13) ^ b;
        return w[0] ^ w[1] ^ w[2] ^ w[3];
    }
};

struct Mrg32k3aEngine // rocrand_mrg32k3a.h:160-190: g1[0..2], g2[0..2]
{
    static constexpr int      kWords  = 6;
    static constexpr int      kUnroll = 6; // two rotation periods of the three-word components
    static constexpr uint64_t kM1 = 4294967087ull, kM2 = 4294944443ull;
    uint32_t                  w[kWords];
    // t < 2 m: t mod m, with the comparison and subtraction on 32-bit words (t - m < 2^32)
    __host__ __device__ __forceinline__ static uint32_t sub_once(uint64_t t, uint32_t m)
    {
        const uint32_t lo = static_cast<uint32_t>(t);
        return (static_cast<uint32_t>(t >> 32) != 0u || lo >= m) ? lo - m : lo;
    }
    // p < 2^54: 2^32 = 209 (mod m1) folds p below 2^33 < 2 m1
    __host__ __device__ __forceinline__ static uint32_t mod_m1(uint64_t p)
    {
        return sub_once(209ull * (p >> 32) + (p & 0xffffffffull), static_cast<uint32_t>(kM1));
    }
    // p < 2^54: two folds by 2^32 = 22853 (mod m2) bring p below 2^33 < 2 m2
    __host__ __device__ __forceinline__ static uint32_t mod_m2(uint64_t p)
    {
        p = 22853ull * (p >> 32) + (p & 0xffffffffull);
        return sub_once(22853ull * (p >> 32) + (p & 0xffffffffull), static_cast<uint32_t>(kM2));
    }
    __host__ __device__ __forceinline__ uint32_t next()
    {
        const uint32_t p1 = mod_m1(1403580ull * w[1] + 810728ull * static_cast<uint32_t>(static_cast<uint32_t>(kM1) - w[0]));
        w[0] = w[1];
        w[1] = w[2];
        w[2] = p1;
        const uint32_t p2 = mod_m2(527612ull * w[5] + 1370589ull * static_cast<uint32_t>(static_cast<uint32_t>(kM2) - w[3]));
        w[3] = w[4];
        w[4] = w[5];
        w[5] = p2;
        return (p1 - p2) + (p1 <= p2 ? static_cast<uint32_t>(kM1) : 0u);
    }
};

struct Mrg31k3pEngine // rocrand_mrg31k3p.h:155-185: x1[0..2], x2[0..2]
{
    static constexpr int      kWords  = 6;
    static constexpr int      kUnroll = 6; // two rotation periods of the three-word components
    static constexpr uint32_t kM1 = 2147483647u, kM2 = 2147462579u;
    uint32_t                  w[kWords];
    __host__ __device__ __forceinline__ uint32_t next()
    {
        uint32_t t = (((w[1] & 511u) << 22) + (w[1] >> 9)) + (((w[2] & 16777215u) << 7) + (w[2] >> 24));
        t -= (t >= kM1) ? kM1 : 0u;
        t += w[2];
        t -= (t >= kM1) ? kM1 : 0u;
        w[2] = w[1];
        w[1] = w[0];
        w[0] = t;
        t    = (((w[3] & 65535u) << 15) + 21069u * (w[3] >> 16));
        t -= (t >= kM2) ? kM2 : 0u;
        t += ((w[5] & 65535u) << 15);
        t -= (t >= kM2) ? kM2 : 0u;
        t += 21069u * (w[5] >> 16);
        t -= (t >= kM2) ? kM2 : 0u;
        t += w[5];
        t -= (t >= kM2) ? kM2 : 0u;
        w[5] = w[4];
        w[4] = w[3];
        w[3] = t;
        return w[0] - w[3] + (w[0] <= w[3] ? kM1 : 0u);
    }
};

// ---- initialisation: engine e = J^e * base[e < start] ----

template<int N>
__host__ __device__ __forceinline__ void gf2_apply(const uint32_t* __restrict__ m, uint32_t* x)
{
    uint32_t y[N];
#pragma unroll
    for(int k = 0; k < N; k++)
        y[k] = 0;
#pragma unroll
    for(int i = 0; i < N; i++)
    {
        const uint32_t xi = x[i];
#pragma unroll 8
        for(int b = 0; b < 32; b++)
        {
            const uint32_t  mask = 0u - ((xi >> b) & 1u);
            const uint32_t* row  = m + (i * 32 + b) * N;
#pragma unroll
            for(int k = 0; k < N; k++)
                y[k] ^= mask & ld_ro(row + k);
        }
    }
#pragma unroll
    for(int k = 0; k < N; k++)
        x[k] = y[k];
}

__host__ __device__ __forceinline__ void mod_apply(const uint64_t* __restrict__ a, uint64_t m, uint32_t* x)
{
    uint32_t y[3];
#pragma unroll
    for(int r = 0; r < 3; r++)
    {
        uint64_t s = 0;
#pragma unroll
        for(int c = 0; c < 3; c++)
            s += (ld_ro(reinterpret_cast<const unsigned long long*>(a) + r * 3 + c) * x[c]) % m;
        y[r] = static_cast<uint32_t>(s % m);
    }
#pragma unroll
    for(int r = 0; r < 3; r++)
        x[r] = y[r];
}

// XORWOW subsequence jumps by polynomial.  Engine e of a fresh generator is the base state
// moved by e subsequences, J^e = A^(e 2^67) with A the 160-bit xorshift step; J^e = p_e(A)
// for a polynomial p_e of degree < 160 (derived at build time, make_xorwow_jump.c), and
// A^k s is the window (s_k .. s_k+4) of the word sequence that continues s.  So engine e's
// words 0..4 are the XOR of the windows k over the set coefficients k of p_e: with the
// 164-word sequence of the base, no matrix is needed.  The windows are grouped four
// coefficients at a time: table entry (g, v) = XOR of the windows 4g + b over the set bits
// b of v (g < 40, v < 16), built once per base in shared memory, so one jump is 40 table
// reads, conflict-free (a warp's 16 possible entries of group g are 16 consecutive ones).
constexpr int kXorwowSeqWords = 164;
constexpr int kXorwowGroups   = 40;

struct XorwowJumpTable
{
    uint2    w01[kXorwowGroups * 16]; // words 0, 1
    uint2    w23[kXorwowGroups * 16]; // words 2, 3
    uint32_t w4[kXorwowGroups * 16];  // word 4
};

// Builds the table of one base from its word sequence (any memory space the block can
// read); called by all `nthreads` threads of the block, which synchronise afterwards.
__host__ __device__ __forceinline__ void xorwow_build_jump_table(XorwowJumpTable& t, const uint32_t* seq,
                                                        uint32_t tid, uint32_t nthreads)
{
    for(uint32_t i = tid; i < kXorwowGroups * 16; i += nthreads)
    {
        const uint32_t g = i >> 4, v = i & 15u;
        uint32_t       y[5] = {0u, 0u, 0u, 0u, 0u};
#pragma unroll
        for(int b = 0; b < 4; b++)
        {
            if((v >> b) & 1u)
            {
#pragma unroll
                for(int j = 0; j < 5; j++)
                    y[j] ^= seq[4 * g + b + j];
            }
        }
        t.w01[i] = make_uint2(y[0], y[1]);
        t.w23[i] = make_uint2(y[2], y[3]);
        t.w4[i]  = y[4];
    }
}

// x[0..4] <- J^e of the table's base; polys = the build-time table, word-major with stride
// kStatefulEngines.  The Weyl word is left as it is (a subsequence jump keeps it).
__host__ __device__ __forceinline__ void xorwow_jump(const XorwowJumpTable& t, const uint32_t* __restrict__ polys,
                                            uint32_t e, uint32_t* x)
{
    uint32_t c[5];
#pragma unroll
    for(int j = 0; j < 5; j++)
        c[j] = ld_ro(polys + static_cast<size_t>(j) * kStatefulEngines + e);
    uint32_t y0 = 0u, y1 = 0u, y2 = 0u, y3 = 0u, y4 = 0u;
#pragma unroll
    for(int g = 0; g < kXorwowGroups; g++)
    {
        const uint32_t i = 16u * g + ((c[g >> 3] >> (4 * (g & 7))) & 15u);
        const uint2    a = t.w01[i];
        const uint2    b = t.w23[i];
        y0 ^= a.x;
        y1 ^= a.y;
        y2 ^= b.x;
        y3 ^= b.y;
        y4 ^= t.w4[i];
    }
    x[0] = y0;
    x[1] = y1;
    x[2] = y2;
    x[3] = y3;
    x[4] = y4;
}

template<class T, unsigned N>
__host__ __device__ __forceinline__ void store_small(unsigned char* p, const T (&v)[N])
{
    constexpr unsigned VB = sizeof(T) * N;
#if !defined(__CUDA_ARCH__)
    memcpy(p, v, VB);
#else
    if constexpr(VB == 4)
    {
        uint32_t w;
        memcpy(&w, v, 4);
        __stcs(reinterpret_cast<unsigned int*>(p), w);
    }
    else if constexpr(VB == 8)
    {
        uint2 w;
        memcpy(&w, v, 8);
        __stcs(reinterpret_cast<uint2*>(p), w);
    }
    else
    {
        static_assert(VB == 16, "vector size");
        uint4 w;
        memcpy(&w, v, 16);
        __stcs(reinterpret_cast<uint4*>(p), w);
    }
#endif
}

} // namespace rb200
