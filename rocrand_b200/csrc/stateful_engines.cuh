// stateful_engines.cuh -- device step functions of the XORWOW, MRG32k3a, MRG31k3p and
// LFSR113 engines, their jump-table application and small vector stores; shared by the
// per-generator kernels (stateful.cu) and the batched fill (batch.cu).
#pragma once

#include "common.hpp"

#include <cstring>

namespace rb200
{

// ---- engines (device step functions; the state is NW 32-bit words) ----

struct XorwowEngine // rocrand_xorwow.h:165-177
{
    static constexpr int kWords = 6; // x[0..4], d
    static constexpr int kGf2   = 5; // words covered by the jump matrices
    uint32_t             w[kWords];
    __device__ __forceinline__ uint32_t next()
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
    static constexpr int kWords = 4;
    static constexpr int kGf2   = 4;
    uint32_t             w[kWords];
    __device__ __forceinline__ uint32_t next()
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
    static constexpr int      kWords = 6;
    static constexpr uint64_t kM1 = 4294967087ull, kM2 = 4294944443ull;
    uint32_t                  w[kWords];
    __device__ __forceinline__ static uint64_t mod_m1(uint64_t p)
    {
        p = 209ull * (p >> 32) + (p & 0xffffffffull);
        return p >= kM1 ? p - kM1 : p;
    }
    __device__ __forceinline__ static uint64_t mod_m2(uint64_t p)
    {
        p = 22853ull * (p >> 32) + (p & 0xffffffffull);
        p = 22853ull * (p >> 32) + (p & 0xffffffffull);
        return p >= kM2 ? p - kM2 : p;
    }
    __device__ __forceinline__ uint32_t next()
    {
        const uint32_t p1 = static_cast<uint32_t>(mod_m1(
            1403580ull * w[1] + 810728ull * static_cast<uint32_t>(static_cast<uint32_t>(kM1) - w[0])));
        w[0] = w[1];
        w[1] = w[2];
        w[2] = p1;
        const uint32_t p2 = static_cast<uint32_t>(mod_m2(
            527612ull * w[5] + 1370589ull * static_cast<uint32_t>(static_cast<uint32_t>(kM2) - w[3])));
        w[3] = w[4];
        w[4] = w[5];
        w[5] = p2;
        return (p1 - p2) + (p1 <= p2 ? static_cast<uint32_t>(kM1) : 0u);
    }
};

struct Mrg31k3pEngine // rocrand_mrg31k3p.h:155-185: x1[0..2], x2[0..2]
{
    static constexpr int      kWords = 6;
    static constexpr uint32_t kM1 = 2147483647u, kM2 = 2147462579u;
    uint32_t                  w[kWords];
    __device__ __forceinline__ uint32_t next()
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
__device__ __forceinline__ void gf2_apply(const uint32_t* __restrict__ m, uint32_t* x)
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
                y[k] ^= mask & __ldg(row + k);
        }
    }
#pragma unroll
    for(int k = 0; k < N; k++)
        x[k] = y[k];
}

__device__ __forceinline__ void mod_apply(const uint64_t* __restrict__ a, uint64_t m, uint32_t* x)
{
    uint32_t y[3];
#pragma unroll
    for(int r = 0; r < 3; r++)
    {
        uint64_t s = 0;
#pragma unroll
        for(int c = 0; c < 3; c++)
            s += (__ldg(reinterpret_cast<const unsigned long long*>(a) + r * 3 + c) * x[c]) % m;
        y[r] = static_cast<uint32_t>(s % m);
    }
#pragma unroll
    for(int r = 0; r < 3; r++)
        x[r] = y[r];
}

// y = M x for one 160x160 GF(2) matrix (column-wise: column i = image of input bit i, 5
// words at m + 5 i) and one x held identically by all 32 lanes of a warp: lane l folds the
// columns of bits l, 32+l, ..., 128+l, then the partial results are XOR-reduced across the
// warp.  25 loads and 25 shuffles per lane instead of 160 x 5 loads.
__device__ __forceinline__ void gf2_apply_warp(const uint32_t* __restrict__ m, uint32_t* x)
{
    const uint32_t l = threadIdx.x & 31u;
    uint32_t       y[5] = {0u, 0u, 0u, 0u, 0u};
#pragma unroll
    for(int w = 0; w < 5; w++)
    {
        const uint32_t  mask = 0u - ((x[w] >> l) & 1u);
        const uint32_t* col  = m + (32u * w + l) * 5u;
#pragma unroll
        for(int k = 0; k < 5; k++)
            y[k] ^= mask & __ldg(col + k);
    }
#pragma unroll
    for(int k = 0; k < 5; k++)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            y[k] ^= __shfl_xor_sync(0xffffffffu, y[k], o);
        x[k] = y[k];
    }
}

// Lane tables of XORWOW seeding: J^r for r = 0..63 (J = one subsequence, 2^67 steps),
// stored [input bit i][word k][r] so that a warp whose lanes apply different r reads
// consecutive words.
constexpr uint32_t kXorwowLaneJumps = 64;

// The XORWOW engine e of a generator whose engines start from `x` (words 0..4 jumped, the
// Weyl word 5 kept): x <- J^e x.  Must be called by all 32 lanes of the warp together
// (it synchronises them).  e = 64 q + r: when the lanes share q and x (shared_base in every
// lane), J^(64 q) is applied by the warp together (radix-4 digits 3..8) and J^r by each lane
// from the lane table; otherwise each lane applies its own 9 digits.
__device__ __forceinline__ void xorwow_seed(uint32_t* x, uint32_t e, const uint32_t* __restrict__ digits,
                                            const uint32_t* __restrict__ lanes, bool shared_base)
{
    constexpr size_t msize = 5 * 32 * 5;
    const uint32_t   q     = e >> 6;
    const uint32_t   q0    = __shfl_sync(0xffffffffu, q, 0);
    if(!__all_sync(0xffffffffu, shared_base && q == q0))
    {
        for(int p = 0; p < 9; p++)
        {
            const uint32_t d = (e >> (2 * p)) & 3u;
            if(d)
                gf2_apply<5>(digits + (static_cast<size_t>(p) * 3 + (d - 1)) * msize, x);
        }
        return;
    }
    for(int p = 3; p < 9; p++)
    {
        const uint32_t d = (q >> (2 * (p - 3))) & 3u; // the same in every lane
        if(d)
            gf2_apply_warp(digits + (static_cast<size_t>(p) * 3 + (d - 1)) * msize, x);
    }
    // x is the same in every lane here, so the loop visits only its set bits, uniformly
    const uint32_t r = e & 63u;
    uint32_t       y[5] = {0u, 0u, 0u, 0u, 0u};
#pragma unroll
    for(int w = 0; w < 5; w++)
    {
        uint32_t bits = x[w];
        while(bits)
        {
            const int       b   = __ffs(bits) - 1;
            const uint32_t* row = lanes + static_cast<size_t>((32 * w + b) * 5) * kXorwowLaneJumps + r;
            bits &= bits - 1;
#pragma unroll
            for(int k = 0; k < 5; k++)
                y[k] ^= __ldg(row + k * kXorwowLaneJumps);
        }
    }
#pragma unroll
    for(int k = 0; k < 5; k++)
        x[k] = y[k];
}

template<class T, unsigned N>
__device__ __forceinline__ void store_small(unsigned char* p, const T (&v)[N])
{
    constexpr unsigned VB = sizeof(T) * N;
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
}

} // namespace rb200
