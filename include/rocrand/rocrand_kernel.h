/*
 * rocrand_kernel.h -- device API of librocrand (B200 build): generator states and
 * distribution functions called from inside user kernels.
 *
 * Drop-in for the reference's device API (library/include/rocrand/rocrand_kernel.h and the
 * engine and distribution headers it includes) for these states:
 *   rocrand_state_philox4x32_10, rocrand_state_xorwow, rocrand_state_mrg32k3a,
 *   rocrand_state_mrg31k3p, rocrand_state_lfsr113, rocrand_state_mtgp32 (block-wide),
 *   rocrand_state_threefry2x32_20, rocrand_state_threefry2x64_20,
 *   rocrand_state_threefry4x32_20, rocrand_state_threefry4x64_20,
 *   rocrand_state_sobol32, rocrand_state_scrambled_sobol32,
 *   rocrand_state_sobol64, rocrand_state_scrambled_sobol64;
 * with rocrand_init, rocrand / rocrand2 / rocrand4, skipahead{,_subsequence,_sequence},
 * rocrand_uniform{,2,4}{,_double}, rocrand_normal{,2,4}{,_double},
 * rocrand_log_normal{,2,4}{,_double}, rocrand_poisson{,4} and rocrand_discrete{,4} as the
 * reference defines them for each state.
 *
 * Values: every function returns what the reference's function of the same name returns for
 * the same state, compiled for the same GPU with the same flags.  To that end each one takes
 * its inputs from the engine in the same order and evaluates the same arithmetic
 * expressions (so the compiler contracts the same multiply-adds); on the device the
 * Box-Muller transforms use __sincosf / sincospi with logf / log, on the host sinf / cosf /
 * sin / cos, as the reference's two builds do.  Reference behaviours kept on purpose are
 * noted where they occur (the cached second Box-Muller double is returned through a float,
 * 64-bit engines feed some float transforms only their low 32 bits, ...).
 *
 * Requires nvcc (the MRG skip-ahead matrices are __device__ arrays).
 */
#ifndef ROCRAND_KERNEL_H_
#define ROCRAND_KERNEL_H_

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math.h>

#include "rocrand/rocrand.h"
#include "rocrand/rocrand_b200_jump_tables.h"
#include "rocrand/rocrand_discrete_types.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ROCRAND_B200_FN __forceinline__ __host__ __device__

/* Conversion constants, the same binary values as library/include/rocrand/rocrand_common.h:24-38. */
#define ROCRAND_2POW16_INV (1.5258789e-05f)
#define ROCRAND_2POW16_INV_2PI (9.58738e-05f)
#define ROCRAND_2POW32_INV (2.3283064e-10f)
#define ROCRAND_2POW32_INV_DOUBLE (2.3283064365386963e-10)
#define ROCRAND_2POW64_INV (5.4210109e-20f)
#define ROCRAND_2POW64_INV_DOUBLE (5.4210108624275221700372640043497e-20)
#define ROCRAND_2POW32_INV_2PI (1.46291807e-09f)
#define ROCRAND_2POW53_INV_DOUBLE (1.1102230246251565e-16)
#define ROCRAND_PI (3.141592653f)
#define ROCRAND_PI_DOUBLE (3.1415926535897932)
#define ROCRAND_2PI (6.2831855f)
#define ROCRAND_SQRT2 (1.4142135f)
#define ROCRAND_SQRT2_DOUBLE (1.4142135623730951)

// default seeds (rocrand_philox4x32_10.h:73, rocrand_xorwow.h:35, rocrand_mrg32k3a.h:49,
// rocrand_mrg31k3p.h:44, rocrand_lfsr113.h:33-42); the C++ wrapper's engines default to them
#define ROCRAND_PHILOX4x32_DEFAULT_SEED 0xdeadbeefdeadbeefULL
#define ROCRAND_XORWOW_DEFAULT_SEED 0ULL
#define ROCRAND_MRG32K3A_DEFAULT_SEED 12345ULL
#define ROCRAND_MRG31K3P_DEFAULT_SEED 12345ULL
#define ROCRAND_LFSR113_DEFAULT_SEED_X 2
#define ROCRAND_LFSR113_DEFAULT_SEED_Y 8
#define ROCRAND_LFSR113_DEFAULT_SEED_Z 16
#define ROCRAND_LFSR113_DEFAULT_SEED_W 128

namespace rocrand_b200_detail
{

// ---------------------------------------------------------------------------------------
// Box-Muller cache of the states that keep one (rocrand_common.h:113-146).  The double
// getter returns through a float, as the reference's does.

template<class S>
ROCRAND_B200_FN bool bm_has_float(const S* s)
{
    return s->boxmuller_float_state != 0;
}
template<class S>
ROCRAND_B200_FN float bm_take_float(S* s)
{
    s->boxmuller_float_state = 0;
    return s->boxmuller_float;
}
template<class S>
ROCRAND_B200_FN void bm_keep_float(S* s, float f)
{
    s->boxmuller_float_state = 1;
    s->boxmuller_float       = f;
}
template<class S>
ROCRAND_B200_FN bool bm_has_double(const S* s)
{
    return s->boxmuller_double_state != 0;
}
template<class S>
ROCRAND_B200_FN float bm_take_double(S* s)
{
    s->boxmuller_double_state = 0;
    return static_cast<float>(s->boxmuller_double);
}
template<class S>
ROCRAND_B200_FN void bm_keep_double(S* s, double d)
{
    s->boxmuller_double_state = 1;
    s->boxmuller_double       = d;
}

// ---------------------------------------------------------------------------------------
// Conversions (rocrand_uniform.h:62-160).

ROCRAND_B200_FN float to_float(unsigned int v)
{
    return ROCRAND_2POW32_INV + (v * ROCRAND_2POW32_INV);
}
ROCRAND_B200_FN float to_float(unsigned long long v)
{
    return ROCRAND_2POW32_INV + (v >> 32) * ROCRAND_2POW32_INV;
}
ROCRAND_B200_FN float4 to_float4(uint4 v)
{
    return float4{ROCRAND_2POW32_INV + (v.x * ROCRAND_2POW32_INV),
                  ROCRAND_2POW32_INV + (v.y * ROCRAND_2POW32_INV),
                  ROCRAND_2POW32_INV + (v.z * ROCRAND_2POW32_INV),
                  ROCRAND_2POW32_INV + (v.w * ROCRAND_2POW32_INV)};
}
ROCRAND_B200_FN double to_double(unsigned int v)
{
    return ROCRAND_2POW32_INV_DOUBLE + (v * ROCRAND_2POW32_INV_DOUBLE);
}
// 53 bits from two words: the low word, then the top 21 bits of the second
ROCRAND_B200_FN double to_double(unsigned int v1, unsigned int v2)
{
    const unsigned long long v = static_cast<unsigned long long>(v1)
                                 | (static_cast<unsigned long long>(v2 >> 11) << 32);
    return ROCRAND_2POW53_INV_DOUBLE + (v * ROCRAND_2POW53_INV_DOUBLE);
}
ROCRAND_B200_FN double to_double(unsigned long long v)
{
    return ROCRAND_2POW53_INV_DOUBLE + ((v >> 11) * ROCRAND_2POW53_INV_DOUBLE);
}

// ---------------------------------------------------------------------------------------
// Normal transforms (rocrand_normal.h:51-236).

ROCRAND_B200_FN float2 box_muller(unsigned int x, unsigned int y)
{
    float2 r;
    float  u = ROCRAND_2POW32_INV + (x * ROCRAND_2POW32_INV);
    float  v = ROCRAND_2POW32_INV_2PI + (y * ROCRAND_2POW32_INV_2PI);
    float  s = sqrtf(-2.0f * logf(u));
#if defined(__CUDA_ARCH__)
    __sincosf(v, &r.x, &r.y);
    r.x *= s;
    r.y *= s;
#else
    r.x = sinf(v) * s;
    r.y = cosf(v) * s;
#endif
    return r;
}

ROCRAND_B200_FN float2 box_muller(unsigned long long v)
{
    return box_muller(static_cast<unsigned int>(v), static_cast<unsigned int>(v >> 32));
}

ROCRAND_B200_FN double2 box_muller_double(uint4 v)
{
    double2                  r;
    const unsigned long long v1 = static_cast<unsigned long long>(v.x)
                                  ^ (static_cast<unsigned long long>(v.y) << (53 - 32));
    double                   u  = ROCRAND_2POW53_INV_DOUBLE + (v1 * ROCRAND_2POW53_INV_DOUBLE);
    const unsigned long long v2 = static_cast<unsigned long long>(v.z)
                                  ^ (static_cast<unsigned long long>(v.w) << (53 - 32));
    double w = (ROCRAND_2POW53_INV_DOUBLE * 2.0) + (v2 * (ROCRAND_2POW53_INV_DOUBLE * 2.0));
    double s = sqrt(-2.0 * log(u));
#if defined(__CUDA_ARCH__)
    sincospi(w, &r.x, &r.y);
    r.x *= s;
    r.y *= s;
#else
    r.x = sin(w * ROCRAND_PI_DOUBLE) * s;
    r.y = cos(w * ROCRAND_PI_DOUBLE) * s;
#endif
    return r;
}

ROCRAND_B200_FN double2 box_muller_double(ulonglong2 v)
{
    return box_muller_double(make_uint4(static_cast<unsigned int>(v.x), static_cast<unsigned int>(v.x >> 32),
                                        static_cast<unsigned int>(v.y), static_cast<unsigned int>(v.y >> 32)));
}

ROCRAND_B200_FN float erfinv_f(float x)
{
    float tt1, tt2, lnx, sgn;
    sgn = (x < 0.0f) ? -1.0f : 1.0f;
    x   = (1.0f - x) * (1.0f + x);
    lnx = logf(x);
    if(isnan(lnx))
        return 1.0f;
    else if(isinf(lnx))
        return 0.0f;
    tt1 = 2.0f / (ROCRAND_PI * 0.147f) + 0.5f * lnx;
    tt2 = 1.0f / (0.147f) * lnx;
    return (sgn * sqrtf(-tt1 + sqrtf(tt1 * tt1 - tt2)));
}

ROCRAND_B200_FN double erfinv_d(double x)
{
    double tt1, tt2, lnx, sgn;
    sgn = (x < 0.0) ? -1.0 : 1.0;
    x   = (1.0 - x) * (1.0 + x);
    lnx = log(x);
    if(isnan(lnx))
        return 1.0;
    else if(isinf(lnx))
        return 0.0;
    tt1 = 2.0 / (ROCRAND_PI_DOUBLE * 0.147) + 0.5 * lnx;
    tt2 = 1.0 / (0.147) * lnx;
    return (sgn * sqrt(-tt1 + sqrt(tt1 * tt1 - tt2)));
}

// the inverse-erf normal of one word
template<class W>
ROCRAND_B200_FN float normal_inv(W x)
{
    float p = to_float(x);
    float v = ROCRAND_SQRT2 * erfinv_f(2.0f * p - 1.0f);
    return v;
}
template<class W>
ROCRAND_B200_FN double normal_inv_double(W x)
{
    double p = to_double(x);
    double v = ROCRAND_SQRT2 * erfinv_d(2.0 * p - 1.0);
    return v;
}

ROCRAND_B200_FN float4 box_muller4(uint4 v)
{
    float2 r1 = box_muller(v.x, v.y);
    float2 r2 = box_muller(v.z, v.w);
    return float4{r1.x, r1.y, r2.x, r2.y};
}

// ---------------------------------------------------------------------------------------
// Poisson (rocrand_poisson.h:36-204): multiplication of uniforms below lambda = 64,
// Atkinson's PA rejection up to 4000, the normal approximation above; the inversion
// sampler (ITR) for the engines the reference gives it.

constexpr double kPoissonSmall = 64.0;
constexpr double kPoissonHuge  = 4000.0;

template<class S>
ROCRAND_B200_FN unsigned int poisson_small(S state, double lambda)
{
    const double limit   = exp(-lambda);
    unsigned int k       = 0;
    double       product = 1.0;
    do
    {
        k++;
        product *= rocrand_uniform_double(state);
    }
    while(product > limit);
    return k - 1;
}

// log Gamma(x) by the Lanczos approximation with g = 7, n = 9 (published coefficients)
ROCRAND_B200_FN double lgamma_lanczos(const double x)
{
    const double z    = x - 1.0;
    const int    g    = 7;
    const double c[9] = {0.99999999999980993227684700473478,  676.520368121885098567009190444019,
                         -1259.13921672240287047156078755283, 771.3234287776530788486528258894,
                         -176.61502916214059906584551354,     12.507343278686904814458936853,
                         -0.13857109526572011689554707,       9.984369578019570859563e-6,
                         1.50563273514931155834e-7};
    double       sum  = 0.0;
#pragma unroll
    for(int i = 8; i > 0; i--)
        sum += c[i] / (z + i);
    sum += c[0];
    const double log_sqrt_2_pi = 0.9189385332046727418;
    const double e             = 2.718281828459045090796;
    return (log_sqrt_2_pi + log(sum) - g) + (z + 0.5) * log((z + g + 0.5) / e);
}

template<class S>
ROCRAND_B200_FN unsigned int poisson_large(S state, double lambda)
{
    const double c          = 0.767 - 3.36 / lambda;
    const double beta       = ROCRAND_PI_DOUBLE / sqrt(3.0 * lambda);
    const double alpha      = beta * lambda;
    const double k          = log(c) - lambda - log(beta);
    const double log_lambda = log(lambda);
    while(true)
    {
        const double u = rocrand_uniform_double(state);
        const double x = (alpha - log((1.0 - u) / u)) / beta;
        const double n = floor(x + 0.5);
        if(n < 0)
            continue;
        const double v   = rocrand_uniform_double(state);
        const double y   = alpha - beta * x;
        const double t   = 1.0 + exp(y);
        const double lhs = y + log(v / (t * t));
        const double rhs = k + n * log_lambda - lgamma_lanczos(n + 1.0);
        if(lhs <= rhs)
            return static_cast<unsigned int>(n);
    }
}

template<class S>
ROCRAND_B200_FN unsigned int poisson_huge(S state, double lambda)
{
    const double n = rocrand_normal_double(state);
    return static_cast<unsigned int>(round(sqrt(lambda) * n + lambda));
}

template<class S>
ROCRAND_B200_FN unsigned int poisson_rejection(S state, double lambda)
{
    if(lambda < kPoissonSmall)
        return poisson_small(state, lambda);
    else if(lambda <= kPoissonHuge)
        return poisson_large(state, lambda);
    else
        return poisson_huge(state, lambda);
}

// Inversion with the cumulative sum rescaled every 500 units of lambda (Kemp's ITR).  The
// reference computes the segment bound once (rocrand_poisson.h:138-168), so for 500 < lambda
// < 1000 it scales by e^-1000 instead of e^-lambda and its search runs until k wraps around
// 2^32; here the bound moves with the segment.  Results are the reference's for lambda <= 500
// (one segment) and the correct inversion above.
template<class S>
ROCRAND_B200_FN unsigned int poisson_itr(S state, double lambda)
{
    double       L;
    double       x  = 1.0;
    double       y  = 1.0;
    unsigned int k  = 0;
    int          pw = 0;
    double       u  = rocrand_uniform_double(state) - ROCRAND_2POW32_INV_DOUBLE / 2.0;
    double       ex = exp(-500.0);
    do
    {
        const double upow = pw + 500.0;
        if(lambda > upow)
            L = ex;
        else
            L = exp((double)(pw - lambda));
        x *= L;
        y *= L;
        pw += 500;
        while(u > y)
        {
            k++;
            x *= ((double)lambda / (double)k);
            y += x;
        }
    }
    while((double)pw < lambda);
    return k;
}

template<class S>
ROCRAND_B200_FN unsigned int poisson_inversion(S state, double lambda)
{
    if(lambda < 1000.0)
        return poisson_itr(state, lambda);
    else
        return poisson_huge(state, lambda);
}

// ---------------------------------------------------------------------------------------
// Discrete distributions (rocrand_discrete.h:38-126): alias table or binary search in the
// cumulative table.

ROCRAND_B200_FN unsigned int alias_pick(const double x, const rocrand_discrete_distribution_st& d)
{
    const double       nx  = d.size * x;
    const double       fnx = floor(nx);
    const double       y   = nx - fnx;
    const unsigned int i   = static_cast<unsigned int>(fnx);
    return d.offset + (y < d.probability[i] ? i : d.alias[i]);
}
ROCRAND_B200_FN unsigned int alias_pick(const unsigned int r, const rocrand_discrete_distribution_st& d)
{
    const double x = r * ROCRAND_2POW32_INV_DOUBLE;
    return alias_pick(x, d);
}
ROCRAND_B200_FN unsigned int alias_pick(const unsigned long long r, const rocrand_discrete_distribution_st& d)
{
    const double x = r * ROCRAND_2POW64_INV_DOUBLE;
    return alias_pick(x, d);
}

ROCRAND_B200_FN unsigned int cdf_pick(const double x, const rocrand_discrete_distribution_st& d)
{
    unsigned int lo = 0, hi = d.size - 1;
    do
    {
        const unsigned int mid = (lo + hi) / 2;
        if(x > d.cdf[mid])
            lo = mid + 1;
        else
            hi = mid;
    }
    while(lo != hi);
    return d.offset + lo;
}
ROCRAND_B200_FN unsigned int cdf_pick(const unsigned int r, const rocrand_discrete_distribution_st& d)
{
    const double x = r * ROCRAND_2POW32_INV_DOUBLE;
    return cdf_pick(x, d);
}
ROCRAND_B200_FN unsigned int cdf_pick(const unsigned long long r, const rocrand_discrete_distribution_st& d)
{
    const double x = r * ROCRAND_2POW64_INV_DOUBLE;
    return cdf_pick(x, d);
}

// ---------------------------------------------------------------------------------------
// Counter arithmetic shared by the counter engines.

// the next block of four counters, carries through all words
template<class V>
ROCRAND_B200_FN V bump4(V c)
{
    c.x++;
    auto add = c.x == 0 ? 1 : 0;
    c.y += add;
    add = c.y == 0 ? add : 0;
    c.z += add;
    add = c.z == 0 ? add : 0;
    c.w += add;
    return c;
}

// the four values from substate s on: prev[s..3] then next[0..s-1]
template<class V>
ROCRAND_B200_FN V interleave4(const V prev, const V next, unsigned int s)
{
    switch(s)
    {
        case 1: return V{prev.y, prev.z, prev.w, next.x};
        case 2: return V{prev.z, prev.w, next.x, next.y};
        case 3: return V{prev.w, next.x, next.y, next.z};
        default: return prev;
    }
}

template<class T>
ROCRAND_B200_FN void split_words(T& lo, T& hi, unsigned long long v)
{
    if(sizeof(T) == 4)
    {
        lo = static_cast<T>(v & 0xFFFFFFFFull);
        hi = static_cast<T>((v >> 32) & 0xFFFFFFFFull);
    }
    else
    {
        lo = static_cast<T>(v);
        hi = 0;
    }
}

// ---------------------------------------------------------------------------------------
// ThreeFry rounds (Salmon et al., "Parallel random numbers: as easy as 1, 2, 3", SC11;
// rotation constants of the Random123 distribution, rocrand_threefry{2,4}_impl.h).

template<class T>
ROCRAND_B200_FN T rotl(T x, int d)
{
    constexpr int bits = 8 * sizeof(T);
    return (x << (d & (bits - 1))) | (x >> ((bits - d) & (bits - 1)));
}

template<class T>
ROCRAND_B200_FN T skein_parity()
{
    return sizeof(T) == 4 ? static_cast<T>(0x1BD11BDAu) : static_cast<T>(0x1BD11BDAA9FC1A22ull);
}

template<class T>
ROCRAND_B200_FN int rot2(int i)
{
    constexpr int r32[8] = {13, 15, 26, 6, 17, 29, 16, 24};
    constexpr int r64[8] = {16, 42, 12, 31, 16, 32, 24, 21};
    return sizeof(T) == 4 ? r32[i] : r64[i];
}

template<class T>
ROCRAND_B200_FN int rot4(int i, int j)
{
    constexpr int r32[8][2] = {{10, 26}, {11, 21}, {13, 27}, {23, 5}, {6, 20}, {17, 11}, {25, 10}, {18, 20}};
    constexpr int r64[8][2] = {{14, 16}, {52, 57}, {23, 40}, {5, 37}, {25, 33}, {46, 12}, {58, 22}, {32, 32}};
    return sizeof(T) == 4 ? r32[i][j] : r64[i][j];
}

template<class T, class V>
ROCRAND_B200_FN V threefry2_rounds(V c, V key)
{
    T ks[3];
    ks[2] = skein_parity<T>();
    ks[0] = key.x;
    ks[1] = key.y;
    ks[2] ^= key.x;
    ks[2] ^= key.y;
    V X = c;
    X.x += ks[0];
    X.y += ks[1];
#pragma unroll
    for(unsigned int r = 0; r < 20; r++)
    {
        X.x += X.y;
        X.y = rotl<T>(X.y, rot2<T>(r & 7u));
        X.y ^= X.x;
        if((r & 3u) == 3)
        {
            const unsigned int j = r / 4;
            X.x += ks[(1 + j) % 3];
            X.y += ks[(2 + j) % 3];
            X.y += 1 + j;
        }
    }
    return X;
}

template<class T, class V>
ROCRAND_B200_FN V threefry4_rounds(V c, V key)
{
    T ks[5];
    ks[4] = skein_parity<T>();
    ks[0] = key.x;
    ks[1] = key.y;
    ks[2] = key.z;
    ks[3] = key.w;
    ks[4] ^= key.x;
    ks[4] ^= key.y;
    ks[4] ^= key.z;
    ks[4] ^= key.w;
    V X = c;
    X.x += ks[0];
    X.y += ks[1];
    X.z += ks[2];
    X.w += ks[3];
#pragma unroll
    for(unsigned int r = 0; r < 20; r++)
    {
        const int r0 = rot4<T>(r & 7u, 0), r1 = rot4<T>(r & 7u, 1);
        if((r & 2u) == 0)
        {
            X.x += X.y;
            X.y = rotl<T>(X.y, r0);
            X.y ^= X.x;
            X.z += X.w;
            X.w = rotl<T>(X.w, r1);
            X.w ^= X.z;
        }
        else
        {
            X.x += X.w;
            X.w = rotl<T>(X.w, r0);
            X.w ^= X.x;
            X.z += X.y;
            X.y = rotl<T>(X.y, r1);
            X.y ^= X.z;
        }
        if((r & 3u) == 3)
        {
            const unsigned int j = r / 4;
            X.x += ks[(1 + j) % 5];
            X.y += ks[(2 + j) % 5];
            X.z += ks[(3 + j) % 5];
            X.w += ks[(4 + j) % 5];
            X.w += 1 + j;
        }
    }
    return X;
}

// ---------------------------------------------------------------------------------------
// MRG modular helpers (rocrand_mrg32k3a.h:200-257, rocrand_mrg31k3p.h:186-215).

// one folding step of 2^32 = 209 (mod m1) and one conditional subtraction (not a full
// reduction for every 64-bit input: the seeding relies on exactly this)
ROCRAND_B200_FN unsigned long long m32_fold1(unsigned long long p)
{
    p = 209ull * (p >> 32) + (p & 0xFFFFFFFFull);
    if(p >= 4294967087ull)
        p -= 4294967087ull;
    return p;
}
ROCRAND_B200_FN unsigned long long m32_fold2(unsigned long long p)
{
    p = 22853ull * (p >> 32) + (p & 0xFFFFFFFFull);
    p = 22853ull * (p >> 32) + (p & 0xFFFFFFFFull);
    if(p >= 4294944443ull)
        p -= 4294944443ull;
    return p;
}
template<int C>
ROCRAND_B200_FN unsigned long long m32_fold(unsigned long long p)
{
    return C == 1 ? m32_fold1(p) : m32_fold2(p);
}
// the seeding product of rocrand_mrg32k3a.h:213-225, with its 64-bit wrap
template<int C>
ROCRAND_B200_FN unsigned long long m32_seed_mul(unsigned int i, unsigned long long j)
{
    long long hi = i / 131072;
    long long lo = i - (hi * 131072);
    long long t1 = static_cast<long long>(m32_fold<C>(static_cast<unsigned long long>(hi) * j) * 131072);
    long long t2 = static_cast<long long>(m32_fold<C>(static_cast<unsigned long long>(lo) * j));
    lo           = static_cast<long long>(m32_fold<C>(static_cast<unsigned long long>(t1 + t2)));
    if(lo < 0)
        lo += C == 1 ? 4294967087ll : 4294944443ll;
    return static_cast<unsigned long long>(lo);
}

// s <- A s (mod m) for a row-major 3x3 matrix with entries below m (exact)
template<class A>
ROCRAND_B200_FN void mod_mat_vec(const A* a, unsigned int* s, unsigned long long m)
{
    const unsigned long long x0 = s[0], x1 = s[1], x2 = s[2];
    unsigned long long       y[3];
#pragma unroll
    for(int r = 0; r < 3; r++)
        y[r] = ((a[3 * r] * x0) % m + (a[3 * r + 1] * x1) % m + (a[3 * r + 2] * x2) % m) % m;
    s[0] = static_cast<unsigned int>(y[0]);
    s[1] = static_cast<unsigned int>(y[1]);
    s[2] = static_cast<unsigned int>(y[2]);
}

// s1, s2 <- the matrices of the set bits of n applied in increasing order
template<class A>
ROCRAND_B200_FN void mrg_jump(const A* t1, const A* t2, unsigned long long m1, unsigned long long m2,
                              unsigned long long n, unsigned int* s1, unsigned int* s2)
{
    int i = 0;
    while(n > 0)
    {
        if(n & 1)
        {
            mod_mat_vec(t1 + i, s1, m1);
            mod_mat_vec(t2 + i, s2, m2);
        }
        n >>= 1;
        i += 9;
    }
}

#if defined(__CUDA_ARCH__)
    #define ROCRAND_B200_TABLE(name) (rocrand_b200_detail::name##_d)
#else
    #define ROCRAND_B200_TABLE(name) (rocrand_b200_detail::name##_h)
#endif

// rightmost zero bit of x (0 for all ones, as the reference's device branch returns)
ROCRAND_B200_FN unsigned int low_zero_bit(unsigned int x)
{
#if defined(__CUDA_ARCH__)
    unsigned int z = __ffs(~x);
    return z ? z - 1 : 0;
#else
    if(x == 0)
        return 0;
    unsigned int z = 0;
    while(x & 1u)
    {
        x >>= 1;
        z++;
    }
    return z;
#endif
}
ROCRAND_B200_FN unsigned int low_zero_bit(unsigned long long x)
{
#if defined(__CUDA_ARCH__)
    unsigned int z = __ffsll(~x);
    return z ? z - 1 : 0;
#else
    if(x == 0)
        return 0;
    unsigned int z = 0;
    while(x & 1ull)
    {
        x >>= 1;
        z++;
    }
    return z;
#endif
}

} // namespace rocrand_b200_detail

// =======================================================================================
// States.

/* Philox4x32-10 (rocrand_philox4x32_10.h:87-315): counter (128 bits), key = seed, the
 * current block of four values and the position in it.  A subsequence is 2^64 blocks. */
struct rocrand_state_philox4x32_10
{
    uint4        counter;
    uint4        result;
    uint2        key;
    unsigned int substate;
    unsigned int boxmuller_float_state;
    unsigned int boxmuller_double_state;
    float        boxmuller_float;
    double       boxmuller_double;

    ROCRAND_B200_FN static uint4 block(uint4 c, uint2 k)
    {
        for(int r = 0; r < 10; r++)
        {
            if(r > 0)
            {
                k.x += 0x9E3779B9u;
                k.y += 0xBB67AE85u;
            }
            const unsigned long long p0 = static_cast<unsigned long long>(0xD2511F53u) * c.x;
            const unsigned long long p1 = static_cast<unsigned long long>(0xCD9E8D57u) * c.z;
            c = make_uint4(static_cast<unsigned int>(p1 >> 32) ^ c.y ^ k.x, static_cast<unsigned int>(p1),
                           static_cast<unsigned int>(p0 >> 32) ^ c.w ^ k.y, static_cast<unsigned int>(p0));
        }
        return c;
    }
    // counter += n blocks (the carry of the reference's discard_state)
    ROCRAND_B200_FN void skip_blocks(unsigned long long n)
    {
        const unsigned int lo = static_cast<unsigned int>(n), hi = static_cast<unsigned int>(n >> 32);
        const uint4        t  = counter;
        counter.x += lo;
        counter.y += hi + (counter.x < t.x ? 1 : 0);
        counter.z += (counter.y < t.y ? 1 : 0);
        counter.w += (counter.z < t.z ? 1 : 0);
    }
    ROCRAND_B200_FN void skip_values(unsigned long long offset)
    {
        substate += offset & 3;
        unsigned long long n = offset / 4;
        n += substate < 4 ? 0 : 1;
        substate += substate < 4 ? 0 : -4;
        skip_blocks(n);
    }
    ROCRAND_B200_FN void skip_subsequences(unsigned long long s)
    {
        const unsigned int lo = static_cast<unsigned int>(s), hi = static_cast<unsigned int>(s >> 32);
        const unsigned int t  = counter.z;
        counter.z += lo;
        counter.w += hi + (counter.z < t ? 1 : 0);
    }
    ROCRAND_B200_FN void refresh() { result = block(counter, key); }
    ROCRAND_B200_FN void seed(unsigned long long seed_value, unsigned long long subsequence,
                              unsigned long long offset)
    {
        key                    = make_uint2(static_cast<unsigned int>(seed_value),
                                            static_cast<unsigned int>(seed_value >> 32));
        counter                = make_uint4(0, 0, 0, 0);
        result                 = make_uint4(0, 0, 0, 0);
        substate               = 0;
        boxmuller_float_state  = 0;
        boxmuller_double_state = 0;
        skip_subsequences(subsequence);
        skip_values(offset);
        refresh();
    }
    ROCRAND_B200_FN unsigned int next()
    {
        const unsigned int v = (&result.x)[substate];
        substate++;
        if(substate == 4)
        {
            substate = 0;
            counter  = rocrand_b200_detail::bump4(counter);
            refresh();
        }
        return v;
    }
    ROCRAND_B200_FN uint4 next4()
    {
        const uint4 v = result;
        counter       = rocrand_b200_detail::bump4(counter);
        refresh();
        return rocrand_b200_detail::interleave4(v, result, substate);
    }
};

/* MRG32k3a (rocrand_mrg32k3a.h:45-258): two order-3 recurrences modulo m1 and m2.
 * Subsequences are 2^76 values apart, sequences 2^127. */
struct rocrand_state_mrg32k3a
{
    unsigned int g1[3];
    unsigned int g2[3];
    unsigned int boxmuller_float_state;
    unsigned int boxmuller_double_state;
    float        boxmuller_float;
    double       boxmuller_double;

    static constexpr unsigned long long kM1 = 4294967087ull, kM2 = 4294944443ull;

    ROCRAND_B200_FN unsigned int next()
    {
        const unsigned int p1 = static_cast<unsigned int>(rocrand_b200_detail::m32_fold1(
            1403580ull * g1[1] + 810728ull * static_cast<unsigned int>(static_cast<unsigned int>(kM1) - g1[0])));
        g1[0] = g1[1];
        g1[1] = g1[2];
        g1[2] = p1;
        const unsigned int p2 = static_cast<unsigned int>(rocrand_b200_detail::m32_fold2(
            527612ull * g2[2] + 1370589ull * static_cast<unsigned int>(static_cast<unsigned int>(kM2) - g2[0])));
        g2[0] = g2[1];
        g2[1] = g2[2];
        g2[2] = p2;
        return (p1 - p2) + (p1 <= p2 ? static_cast<unsigned int>(kM1) : 0u);
    }
    ROCRAND_B200_FN void skip_values(unsigned long long n)
    {
        rocrand_b200_detail::mrg_jump(ROCRAND_B200_TABLE(mrg32k3a_a1), ROCRAND_B200_TABLE(mrg32k3a_a2), kM1, kM2,
                                      n, g1, g2);
    }
    ROCRAND_B200_FN void skip_subsequences(unsigned long long n)
    {
        rocrand_b200_detail::mrg_jump(ROCRAND_B200_TABLE(mrg32k3a_a1_sub), ROCRAND_B200_TABLE(mrg32k3a_a2_sub),
                                      kM1, kM2, n, g1, g2);
    }
    ROCRAND_B200_FN void skip_sequences(unsigned long long n)
    {
        rocrand_b200_detail::mrg_jump(ROCRAND_B200_TABLE(mrg32k3a_a1_seq), ROCRAND_B200_TABLE(mrg32k3a_a2_seq),
                                      kM1, kM2, n, g1, g2);
    }
    ROCRAND_B200_FN void seed(unsigned long long s, unsigned long long subsequence, unsigned long long offset)
    {
        if(s == 0)
            s = ROCRAND_MRG32K3A_DEFAULT_SEED;
        const unsigned int x = static_cast<unsigned int>(s) ^ 0x55555555U;
        const unsigned int y = static_cast<unsigned int>((s >> 32) ^ 0xAAAAAAAAU);
        g1[0]                = static_cast<unsigned int>(rocrand_b200_detail::m32_seed_mul<1>(x, s));
        g1[1]                = static_cast<unsigned int>(rocrand_b200_detail::m32_seed_mul<1>(y, s));
        g1[2]                = static_cast<unsigned int>(rocrand_b200_detail::m32_seed_mul<1>(x, s));
        g2[0]                = static_cast<unsigned int>(rocrand_b200_detail::m32_seed_mul<2>(y, s));
        g2[1]                = static_cast<unsigned int>(rocrand_b200_detail::m32_seed_mul<2>(x, s));
        g2[2]                = static_cast<unsigned int>(rocrand_b200_detail::m32_seed_mul<2>(y, s));
        boxmuller_float_state  = 0;
        boxmuller_double_state = 0;
        skip_subsequences(subsequence);
        skip_values(offset);
    }
};

/* MRG31k3p (rocrand_mrg31k3p.h:43-216).  Subsequences are 2^72 values apart, sequences
 * 2^134. */
struct rocrand_state_mrg31k3p
{
    unsigned int x1[3];
    unsigned int x2[3];
    unsigned int boxmuller_float_state;
    unsigned int boxmuller_double_state;
    float        boxmuller_float;
    double       boxmuller_double;

    static constexpr unsigned int kM1 = 2147483647u, kM2 = 2147462579u;

    ROCRAND_B200_FN unsigned int next()
    {
        unsigned int t = (((x1[1] & 511u) << 22) + (x1[1] >> 9)) + (((x1[2] & 16777215u) << 7) + (x1[2] >> 24));
        t -= (t >= kM1) ? kM1 : 0;
        t += x1[2];
        t -= (t >= kM1) ? kM1 : 0;
        x1[2] = x1[1];
        x1[1] = x1[0];
        x1[0] = t;
        t     = (((x2[0] & 65535u) << 15) + 21069u * (x2[0] >> 16));
        t -= (t >= kM2) ? kM2 : 0;
        t += ((x2[2] & 65535u) << 15);
        t -= (t >= kM2) ? kM2 : 0;
        t += 21069u * (x2[2] >> 16);
        t -= (t >= kM2) ? kM2 : 0;
        t += x2[2];
        t -= (t >= kM2) ? kM2 : 0;
        x2[2] = x2[1];
        x2[1] = x2[0];
        x2[0] = t;
        return x1[0] - x2[0] + (x1[0] <= x2[0] ? kM1 : 0);
    }
    ROCRAND_B200_FN void skip_values(unsigned long long n)
    {
        rocrand_b200_detail::mrg_jump(ROCRAND_B200_TABLE(mrg31k3p_a1), ROCRAND_B200_TABLE(mrg31k3p_a2),
                                      static_cast<unsigned long long>(kM1), static_cast<unsigned long long>(kM2), n,
                                      x1, x2);
    }
    ROCRAND_B200_FN void skip_subsequences(unsigned long long n)
    {
        rocrand_b200_detail::mrg_jump(ROCRAND_B200_TABLE(mrg31k3p_a1_sub), ROCRAND_B200_TABLE(mrg31k3p_a2_sub),
                                      static_cast<unsigned long long>(kM1), static_cast<unsigned long long>(kM2), n,
                                      x1, x2);
    }
    ROCRAND_B200_FN void skip_sequences(unsigned long long n)
    {
        rocrand_b200_detail::mrg_jump(ROCRAND_B200_TABLE(mrg31k3p_a1_seq), ROCRAND_B200_TABLE(mrg31k3p_a2_seq),
                                      static_cast<unsigned long long>(kM1), static_cast<unsigned long long>(kM2), n,
                                      x1, x2);
    }
    ROCRAND_B200_FN void seed(unsigned long long s, unsigned long long subsequence, unsigned long long offset)
    {
        if(s == 0)
            s = ROCRAND_MRG31K3P_DEFAULT_SEED;
        const unsigned int x = static_cast<unsigned int>(s ^ 0x55555555U);
        const unsigned int y = static_cast<unsigned int>((s >> 32) ^ 0xAAAAAAAAU);
        // (i * j) mod m with the 64-bit product wrapping (rocrand_mrg31k3p.h:199-211)
        x1[0]                  = static_cast<unsigned int>((x * s) % kM1);
        x1[1]                  = static_cast<unsigned int>((y * s) % kM1);
        x1[2]                  = static_cast<unsigned int>((x * s) % kM1);
        x2[0]                  = static_cast<unsigned int>((y * s) % kM2);
        x2[1]                  = static_cast<unsigned int>((x * s) % kM2);
        x2[2]                  = static_cast<unsigned int>((y * s) % kM2);
        boxmuller_float_state  = 0;
        boxmuller_double_state = 0;
        skip_subsequences(subsequence);
        skip_values(offset);
    }
};

/* XORWOW (rocrand_xorwow.h:60-208): Marsaglia's xorshift160 plus a Weyl counter.  Skips
 * by values and by subsequences (2^67 values) are taken base 4: each nonzero digit d at
 * position i applies the polynomial x^(d 4^i) (or x^(d 4^i 2^67)) modulo the characteristic
 * polynomial of the xorshift step to the state -- the same map as the reference's jump
 * matrices, as 160 steps of a copy of the state and the XOR of the states at the set
 * coefficients. */
struct rocrand_state_xorwow
{
    unsigned int d;
    unsigned int boxmuller_float_state;
    unsigned int boxmuller_double_state;
    float        boxmuller_float;
    double       boxmuller_double;
    unsigned int x[5];

    ROCRAND_B200_FN static void step(unsigned int* v)
    {
        const unsigned int t = v[0] ^ (v[0] >> 2);
        v[0]                 = v[1];
        v[1]                 = v[2];
        v[2]                 = v[3];
        v[3]                 = v[4];
        v[4]                 = (v[4] ^ (v[4] << 4)) ^ (t ^ (t << 1));
    }
    ROCRAND_B200_FN unsigned int next()
    {
        step(x);
        d += 362437;
        return d + x[4];
    }
    // x <- q(A) x for a polynomial q of degree < 160 (5 words)
    ROCRAND_B200_FN void apply(const unsigned int* q)
    {
        unsigned int v[5] = {x[0], x[1], x[2], x[3], x[4]};
        unsigned int y[5] = {0, 0, 0, 0, 0};
        for(int w = 0; w < 5; w++)
        {
            const unsigned int bits = q[w];
            for(int b = 0; b < 32; b++)
            {
                const unsigned int m = 0u - ((bits >> b) & 1u);
#pragma unroll
                for(int k = 0; k < 5; k++)
                    y[k] ^= m & v[k];
                step(v);
            }
        }
#pragma unroll
        for(int k = 0; k < 5; k++)
            x[k] = y[k];
    }
    ROCRAND_B200_FN void jump(const unsigned int* table, unsigned long long n)
    {
        int i = 0;
        while(n > 0)
        {
            const unsigned int dg = static_cast<unsigned int>(n & 3u);
            if(dg)
                apply(table + (3 * i + (dg - 1)) * 5);
            n >>= 2;
            i++;
        }
    }
    ROCRAND_B200_FN void skip_values(unsigned long long offset)
    {
        jump(ROCRAND_B200_TABLE(xorwow_poly), offset);
        d += static_cast<unsigned int>(offset) * 362437;
    }
    ROCRAND_B200_FN void skip_subsequences(unsigned long long subsequence)
    {
        jump(ROCRAND_B200_TABLE(xorwow_poly_sub), subsequence);
    }
    ROCRAND_B200_FN void seed(unsigned long long s, unsigned long long subsequence, unsigned long long offset)
    {
        x[0]                  = 123456789U;
        x[1]                  = 362436069U;
        x[2]                  = 521288629U;
        x[3]                  = 88675123U;
        x[4]                  = 5783321U;
        d                     = 6615241U;
        const unsigned int s0 = static_cast<unsigned int>(s) ^ 0x2c7f967fU;
        const unsigned int s1 = static_cast<unsigned int>(s >> 32) ^ 0xa03697cbU;
        const unsigned int t0 = 1228688033U * s0;
        const unsigned int t1 = 2073658381U * s1;
        x[0] += t0;
        x[1] ^= t0;
        x[2] += t1;
        x[3] ^= t1;
        x[4] += t0;
        d += t1 + t0;
        skip_subsequences(subsequence);
        skip_values(offset);
        boxmuller_float_state  = 0;
        boxmuller_double_state = 0;
    }
};

/* LFSR113 (rocrand_lfsr113.h:40-160): L'Ecuyer's four Tausworthe components.  Skips by
 * values and by subsequences (2^55 values) are taken base 4; each nonzero digit moves every
 * component by its own polynomial: one step (the step ignores the masked low bits of a word,
 * so its image is where the component's minimal polynomial holds), then the XOR of the
 * component's next states at the set coefficients of x^(d 4^i S - 1) mod that polynomial --
 * the same map as the reference's 128x128 jump matrices. */
struct rocrand_state_lfsr113
{
    uint4 z;
    uint4 subsequence; // the seed, kept as the reference's state keeps it

    ROCRAND_B200_FN static unsigned int step_c(int j, unsigned int v)
    {
        unsigned int b;
        switch(j)
        {
            case 0: b = ((v << 6) ^ v) >> 13; return ((v & 4294967294U) << 18) ^ b;
            case 1: b = ((v << 2) ^ v) >> 27; return ((v & 4294967288U) << 2) ^ b;
            case 2: b = ((v << 13) ^ v) >> 21; return ((v & 4294967280U) << 7) ^ b;
            default: b = ((v << 3) ^ v) >> 12; return ((v & 4294967168U) << 13) ^ b;
        }
    }
    ROCRAND_B200_FN unsigned int next()
    {
        unsigned int b;
        b   = (((z.x << 6) ^ z.x) >> 13);
        z.x = (((z.x & 4294967294U) << 18) ^ b);
        b   = (((z.y << 2) ^ z.y) >> 27);
        z.y = (((z.y & 4294967288U) << 2) ^ b);
        b   = (((z.z << 13) ^ z.z) >> 21);
        z.z = (((z.z & 4294967280U) << 7) ^ b);
        b   = (((z.w << 3) ^ z.w) >> 12);
        z.w = (((z.w & 4294967168U) << 13) ^ b);
        return (z.x ^ z.y ^ z.z ^ z.w);
    }
    ROCRAND_B200_FN static unsigned int apply_c(int j, unsigned int q, unsigned int deg, unsigned int v)
    {
        unsigned int y = step_c(j, v), acc = 0;
        for(unsigned int k = 0; k < deg; k++)
        {
            acc ^= (0u - ((q >> k) & 1u)) & y;
            y = step_c(j, y);
        }
        return acc;
    }
    ROCRAND_B200_FN void jump(const unsigned int* table, unsigned long long n)
    {
        const unsigned int* deg = ROCRAND_B200_TABLE(lfsr113_degree);
        int                 i   = 0;
        while(n > 0)
        {
            const unsigned int dg = static_cast<unsigned int>(n & 3u);
            if(dg)
            {
                const unsigned int* q = table + (3 * i + (dg - 1)) * 4;
                z.x                   = apply_c(0, q[0], deg[0], z.x);
                z.y                   = apply_c(1, q[1], deg[1], z.y);
                z.z                   = apply_c(2, q[2], deg[2], z.z);
                z.w                   = apply_c(3, q[3], deg[3], z.w);
            }
            n >>= 2;
            i++;
        }
    }
    ROCRAND_B200_FN void skip_values(unsigned long long n) { jump(ROCRAND_B200_TABLE(lfsr113_poly), n); }
    ROCRAND_B200_FN void skip_subsequences(unsigned int n) { jump(ROCRAND_B200_TABLE(lfsr113_poly_sub), n); }
    ROCRAND_B200_FN void seed(uint4 s, unsigned int sub, unsigned long long offset)
    {
        subsequence = s;
        z           = s;
        skip_subsequences(sub);
        skip_values(offset);
    }
};

/* MTGP32 (rocrand_mtgp32.h): the block generators of Saito and Matsumoto's MTGP with
 * Mersenne exponent 11213.  One state per thread block (its 1024-word ring, ring offset and
 * parameter set), made on the host by rocrand_make_state_mtgp32 from the published
 * parameter sets (rocrand/rocrand_mtgp32_11213.h); rocrand(state) is called by every thread
 * of the block together and gives thread t the value t of the block's next 256 (blockDim.x)
 * values. */
#define MTGP_MEXP 11213
#define MTGP_N 351
#define MTGP_FLOOR_2P 256
#define MTGP_CEIL_2P 512
#define MTGP_TN MTGP_FLOOR_2P
#define MTGP_LS (MTGP_TN * 3)
#define MTGP_BN_MAX 512
#define MTGP_TS 16
#define MTGP_STATE 1024
#define MTGP_MASK 1023

struct mtgp32_params_fast_t
{
    int           mexp;
    int           pos;
    int           sh1;
    int           sh2;
    unsigned int  tbl[16];
    unsigned int  tmp_tbl[16];
    unsigned int  flt_tmp_tbl[16];
    unsigned int  mask;
    unsigned char poly_sha1[21];
};
typedef mtgp32_params_fast_t mtgp32_fast_params;

/* the parameter sets of all blocks, as rocrand_make_constant lays them out in device memory */
struct mtgp32_params
{
    unsigned int pos_tbl[MTGP_BN_MAX];
    unsigned int param_tbl[MTGP_BN_MAX][MTGP_TS];
    unsigned int temper_tbl[MTGP_BN_MAX][MTGP_TS];
    unsigned int single_temper_tbl[MTGP_BN_MAX][MTGP_TS];
    unsigned int sh1_tbl[MTGP_BN_MAX];
    unsigned int sh2_tbl[MTGP_BN_MAX];
    unsigned int mask[1];
};

struct mtgp32_state
{
    int          offset;
    int          id;
    unsigned int status[MTGP_STATE];
};

struct rocrand_state_mtgp32
{
    mtgp32_state m_state;
    unsigned int pos_tbl;
    unsigned int param_tbl[MTGP_TS];
    unsigned int temper_tbl[MTGP_TS];
    unsigned int sh1_tbl;
    unsigned int sh2_tbl;
    unsigned int single_temper_tbl[MTGP_TS];
    unsigned int mask;

    ROCRAND_B200_FN unsigned int recursion(unsigned int x1, unsigned int x2, unsigned int y) const
    {
        unsigned int x = (x1 & mask) ^ x2;
        x ^= x << sh1_tbl;
        y = x ^ (y >> sh2_tbl);
        return y ^ param_tbl[y & 0x0f];
    }
    ROCRAND_B200_FN unsigned int temper(unsigned int v, unsigned int t) const
    {
        t ^= t >> 16;
        t ^= t >> 8;
        return v ^ temper_tbl[t & 0x0f];
    }
#if defined(__CUDACC__)
    // every thread of the block, together
    __device__ __forceinline__ unsigned int next()
    {
        const unsigned int t = threadIdx.x;
        const int          k = m_state.offset;
        const unsigned int r = recursion(m_state.status[(t + k) & MTGP_MASK], m_state.status[(t + k + 1) & MTGP_MASK],
                                         m_state.status[(t + k + pos_tbl) & MTGP_MASK]);
        m_state.status[(t + k + MTGP_N) & MTGP_MASK] = r;
        const unsigned int o = temper(r, m_state.status[(t + k + pos_tbl - 1) & MTGP_MASK]);
        __syncthreads();
        if(t == 0)
            m_state.offset = (m_state.offset + blockDim.x) & MTGP_MASK;
        __syncthreads();
        return o;
    }
#endif
};

namespace rocrand_b200_detail
{
// the seeding of one block's ring (rocrand_mtgp32.h:154-177): a fill byte from the tables,
// the seed and a hidden word, then the Knuth-style recurrence over the 351 words
inline void mtgp32_seed_ring(unsigned int array[], const mtgp32_fast_params* para, unsigned int seed)
{
    const int    size   = para->mexp / 32 + 1;
    unsigned int hidden = para->tbl[4] ^ (para->tbl[8] << 16);
    unsigned int tmp    = hidden;
    tmp += tmp >> 16;
    tmp += tmp >> 8;
    memset(array, tmp & 0xff, sizeof(unsigned int) * size);
    array[0] = seed;
    array[1] = hidden;
    for(int i = 1; i < size; i++)
        array[i] ^= 1812433253u * (array[i - 1] ^ (array[i - 1] >> 30)) + static_cast<unsigned int>(i);
}
} // namespace rocrand_b200_detail

/* Fills n states (device memory) for n blocks from parameter sets params[0..n) and seed
 * (rocrand_mtgp32.h:394-430): block i gets set i and seed (uint)(seed ^ seed >> 32) + i + 1. */
__host__ inline rocrand_status rocrand_make_state_mtgp32(rocrand_state_mtgp32* state, mtgp32_fast_params params[],
                                                         int n, unsigned long long seed)
{
    rocrand_state_mtgp32* h = static_cast<rocrand_state_mtgp32*>(malloc(sizeof(rocrand_state_mtgp32) * n));
    seed                    = seed ^ (seed >> 32);
    if(h == NULL)
        return ROCRAND_STATUS_ALLOCATION_FAILED;
    for(int i = 0; i < n; i++)
    {
        rocrand_b200_detail::mtgp32_seed_ring(h[i].m_state.status, &params[i],
                                              static_cast<unsigned int>(seed) + i + 1);
        h[i].m_state.offset = 0;
        h[i].m_state.id     = i;
        h[i].pos_tbl        = params[i].pos;
        h[i].sh1_tbl        = params[i].sh1;
        h[i].sh2_tbl        = params[i].sh2;
        h[i].mask           = params[0].mask;
        for(int j = 0; j < MTGP_TS; j++)
        {
            h[i].param_tbl[j]         = params[i].tbl[j];
            h[i].temper_tbl[j]        = params[i].tmp_tbl[j];
            h[i].single_temper_tbl[j] = params[i].flt_tmp_tbl[j];
        }
    }
    const cudaError_t e = cudaMemcpy(state, h, sizeof(rocrand_state_mtgp32) * n, cudaMemcpyDefault);
    free(h);
    return e == cudaSuccess ? ROCRAND_STATUS_SUCCESS : ROCRAND_STATUS_ALLOCATION_FAILED;
}

/* Lays the parameter sets of all MTGP_BN_MAX blocks out in p (device memory), for
 * rocrand_mtgp32_set_params (rocrand_mtgp32.h:432-500). */
__host__ inline rocrand_status rocrand_make_constant(const mtgp32_fast_params params[], mtgp32_params* p)
{
    mtgp32_params* h = static_cast<mtgp32_params*>(malloc(sizeof(mtgp32_params)));
    if(h == NULL)
        return ROCRAND_STATUS_ALLOCATION_FAILED;
    h->mask[0] = params[0].mask;
    for(int i = 0; i < MTGP_BN_MAX; i++)
    {
        h->pos_tbl[i] = params[i].pos;
        h->sh1_tbl[i] = params[i].sh1;
        h->sh2_tbl[i] = params[i].sh2;
        for(int j = 0; j < MTGP_TS; j++)
        {
            h->param_tbl[i][j]         = params[i].tbl[j];
            h->temper_tbl[i][j]        = params[i].tmp_tbl[j];
            h->single_temper_tbl[i][j] = params[i].flt_tmp_tbl[j];
        }
    }
    const cudaError_t e = cudaMemcpy(p, h, sizeof(mtgp32_params), cudaMemcpyHostToDevice);
    free(h);
    return e == cudaSuccess ? ROCRAND_STATUS_SUCCESS : ROCRAND_STATUS_ALLOCATION_FAILED;
}

#if defined(__CUDACC__)
/* Block-cooperative copy of a state (e.g. from global into shared memory). */
__device__ __forceinline__ void rocrand_mtgp32_block_copy(rocrand_state_mtgp32* src, rocrand_state_mtgp32* dest)
{
    const unsigned int t = threadIdx.x;
    for(unsigned int i = t; i < MTGP_STATE; i += blockDim.x)
        dest->m_state.status[i] = src->m_state.status[i];
    if(t == 0)
    {
        dest->m_state.offset = src->m_state.offset;
        dest->m_state.id     = src->m_state.id;
        dest->pos_tbl        = src->pos_tbl;
        dest->sh1_tbl        = src->sh1_tbl;
        dest->sh2_tbl        = src->sh2_tbl;
        dest->mask           = src->mask;
    }
    if(t < MTGP_TS)
    {
        dest->param_tbl[t]         = src->param_tbl[t];
        dest->temper_tbl[t]        = src->temper_tbl[t];
        dest->single_temper_tbl[t] = src->single_temper_tbl[t];
    }
    __syncthreads();
}
/* Takes the state's parameter set, number m_state.id, from a rocrand_make_constant table. */
__device__ __forceinline__ void rocrand_mtgp32_set_params(rocrand_state_mtgp32* state, mtgp32_params* params)
{
    const int id   = state->m_state.id;
    state->pos_tbl = params->pos_tbl[id];
    state->sh1_tbl = params->sh1_tbl[id];
    state->sh2_tbl = params->sh2_tbl[id];
    state->mask    = params->mask[0];
    for(int j = 0; j < MTGP_TS; j++)
    {
        state->param_tbl[j]         = params->param_tbl[id][j];
        state->temper_tbl[j]        = params->temper_tbl[id][j];
        state->single_temper_tbl[j] = params->single_temper_tbl[id][j];
    }
}
#endif

/* ThreeFry states (rocrand_threefry{2,4}_impl.h, rocrand_threefry{2x32,2x64,4x32,4x64}_20.h):
 * counter and key vectors of N words of type T, the current block and the position in it. */
template<class T, class V, int N>
struct rocrand_b200_threefry_state
{
    V            counter;
    V            key;
    V            result;
    unsigned int substate;

    ROCRAND_B200_FN V rounds(V c) const
    {
        if constexpr(N == 2)
            return rocrand_b200_detail::threefry2_rounds<T>(c, key);
        else
            return rocrand_b200_detail::threefry4_rounds<T>(c, key);
    }
    ROCRAND_B200_FN void refresh() { result = rounds(counter); }
    ROCRAND_B200_FN V bump(V c) const
    {
        if constexpr(N == 2)
        {
            c.x++;
            T add = c.x == 0 ? 1 : 0;
            c.y += add;
            return c;
        }
        else
        {
            return rocrand_b200_detail::bump4(c);
        }
    }
    ROCRAND_B200_FN void skip_blocks(unsigned long long n)
    {
        T lo, hi;
        rocrand_b200_detail::split_words(lo, hi, n);
        if constexpr(N == 2)
        {
            const T t = counter.x;
            counter.x += lo;
            counter.y += hi + (counter.x < t ? 1 : 0);
        }
        else
        {
            const V t = counter;
            counter.x += lo;
            counter.y += hi + (counter.x < t.x ? 1 : 0);
            counter.z += (counter.y < t.y ? 1 : 0);
            counter.w += (counter.z < t.z ? 1 : 0);
        }
    }
    ROCRAND_B200_FN void skip_values(unsigned long long offset)
    {
        substate += offset & (N - 1);
        unsigned long long n = offset / N;
        n += substate < N ? 0 : 1;
        substate += substate < N ? 0 : -N;
        skip_blocks(n);
    }
    ROCRAND_B200_FN void skip_subsequences(unsigned long long s)
    {
        if constexpr(N == 2)
        {
            counter.y += s;
        }
        else
        {
            T lo, hi;
            rocrand_b200_detail::split_words(lo, hi, s);
            const T t = counter.z;
            counter.z += lo;
            counter.w += hi + (counter.z < t ? 1 : 0);
        }
    }
    ROCRAND_B200_FN void start(V k, unsigned long long subsequence, unsigned long long offset)
    {
        counter  = V{};
        result   = V{};
        substate = 0;
        key      = k;
        skip_subsequences(subsequence);
        skip_values(offset);
        refresh();
        refresh();
    }
    ROCRAND_B200_FN T next()
    {
        const T v = (&result.x)[substate];
        substate++;
        if(substate == N)
        {
            substate = 0;
            counter  = bump(counter);
            refresh();
        }
        return v;
    }
    ROCRAND_B200_FN V next_block()
    {
        const V v = result;
        counter   = bump(counter);
        refresh();
        if constexpr(N == 2)
            return substate == 1 ? V{v.y, result.x} : v;
        else
            return rocrand_b200_detail::interleave4(v, result, substate);
    }
};

/* Sobol states (rocrand_sobol{32,64}.h, rocrand_scrambled_sobol{32,64}.h): the point of
 * index i of one dimension, its 32 or 64 direction vectors (copied into the state), and
 * for the scrambled ones the XOR constant of the dimension. */
template<class T, int B>
struct rocrand_b200_sobol_state
{
    T d;
    T i;
    T vectors[B];

    ROCRAND_B200_FN void start(const T* v, T offset)
    {
        d = 0;
        i = 0;
        for(int k = 0; k < B; k++)
            vectors[k] = v[k];
        jump(offset);
    }
    // point i + offset from its Gray code
    ROCRAND_B200_FN void jump(T offset)
    {
        i += offset;
        const T g = i ^ (i >> 1);
        d         = 0;
        for(int k = 0; k < B; k++)
            d ^= (g & (T(1) << k) ? vectors[k] : 0);
    }
    ROCRAND_B200_FN T next()
    {
        const T p = d;
        d ^= vectors[rocrand_b200_detail::low_zero_bit(i)];
        i++;
        return p;
    }
};

typedef rocrand_b200_threefry_state<unsigned int, uint2, 2>             rocrand_state_threefry2x32_20;
typedef rocrand_b200_threefry_state<unsigned long long, ulonglong2, 2> rocrand_state_threefry2x64_20;
typedef rocrand_b200_threefry_state<unsigned int, uint4, 4>             rocrand_state_threefry4x32_20;
typedef rocrand_b200_threefry_state<unsigned long long, ulonglong4, 4> rocrand_state_threefry4x64_20;

typedef rocrand_b200_sobol_state<unsigned int, 32>       rocrand_state_sobol32;
typedef rocrand_b200_sobol_state<unsigned long long, 64> rocrand_state_sobol64;

struct rocrand_state_scrambled_sobol32
{
    rocrand_state_sobol32 engine;
    unsigned int          scramble_constant;
};
struct rocrand_state_scrambled_sobol64
{
    rocrand_state_sobol64 engine;
    unsigned long long    scramble_constant;
};

// =======================================================================================
// Initialisation, raw values and skip-ahead.

ROCRAND_B200_FN void rocrand_init(const unsigned long long seed, const unsigned long long subsequence,
                                  const unsigned long long offset, rocrand_state_philox4x32_10* state)
{
    state->seed(seed, subsequence, offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned long long seed, const unsigned long long subsequence,
                                  const unsigned long long offset, rocrand_state_mrg32k3a* state)
{
    state->seed(seed, subsequence, offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned long long seed, const unsigned long long subsequence,
                                  const unsigned long long offset, rocrand_state_mrg31k3p* state)
{
    state->seed(seed, subsequence, offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned long long seed, const unsigned long long subsequence,
                                  const unsigned long long offset, rocrand_state_xorwow* state)
{
    state->seed(seed, subsequence, offset);
}
/* LFSR113 takes its four seed words as they are (rocrand_lfsr113.h:167-180) */
ROCRAND_B200_FN void rocrand_init(const uint4 seed, const unsigned int subsequence, rocrand_state_lfsr113* state)
{
    state->seed(seed, subsequence, 0);
}
ROCRAND_B200_FN void rocrand_init(const uint4 seed, const unsigned int subsequence, const unsigned long long offset,
                                  rocrand_state_lfsr113* state)
{
    state->seed(seed, subsequence, offset);
}
/* ThreeFry keys (rocrand_threefry{2x32,2x64,4x32,4x64}_20.h seed()): 2x32 {lo, hi};
 * 2x64 {seed, seed >> 32}; 4x32 and 4x64 {seed, seed >> 16, seed >> 32, seed >> 48}. */
ROCRAND_B200_FN void rocrand_init(const unsigned long long seed, const unsigned long long subsequence,
                                  const unsigned long long offset, rocrand_state_threefry2x32_20* state)
{
    state->start(make_uint2(static_cast<unsigned int>(seed), static_cast<unsigned int>(seed >> 32)), subsequence,
                 offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned long long seed, const unsigned long long subsequence,
                                  const unsigned long long offset, rocrand_state_threefry2x64_20* state)
{
    state->start(ulonglong2{seed, seed >> 32}, subsequence, offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned long long seed, const unsigned long long subsequence,
                                  const unsigned long long offset, rocrand_state_threefry4x32_20* state)
{
    state->start(make_uint4(static_cast<unsigned int>(seed), static_cast<unsigned int>(seed >> 16),
                            static_cast<unsigned int>(seed >> 32), static_cast<unsigned int>(seed >> 48)),
                 subsequence, offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned long long seed, const unsigned long long subsequence,
                                  const unsigned long long offset, rocrand_state_threefry4x64_20* state)
{
    state->start(ulonglong4{seed, seed >> 16, seed >> 32, seed >> 48}, subsequence, offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned int* vectors, const unsigned int offset,
                                  rocrand_state_sobol32* state)
{
    state->start(vectors, offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned long long* vectors, const unsigned int offset,
                                  rocrand_state_sobol64* state)
{
    state->start(vectors, offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned int* vectors, const unsigned int scramble_constant,
                                  const unsigned int offset, rocrand_state_scrambled_sobol32* state)
{
    state->engine.start(vectors, 0);
    state->scramble_constant = scramble_constant;
    state->engine.jump(offset);
}
ROCRAND_B200_FN void rocrand_init(const unsigned long long* vectors, const unsigned long long scramble_constant,
                                  const unsigned int offset, rocrand_state_scrambled_sobol64* state)
{
    state->engine.start(vectors, 0);
    state->scramble_constant = scramble_constant;
    state->engine.jump(offset);
}

ROCRAND_B200_FN unsigned int rocrand(rocrand_state_philox4x32_10* state)
{
    return state->next();
}
ROCRAND_B200_FN uint4 rocrand4(rocrand_state_philox4x32_10* state)
{
    return state->next4();
}
ROCRAND_B200_FN unsigned int rocrand(rocrand_state_xorwow* state)
{
    return state->next();
}
ROCRAND_B200_FN unsigned int rocrand(rocrand_state_lfsr113* state)
{
    return state->next();
}
/* MRG raw values are remapped from [1, m1] to 32 bits (rocrand_mrg32k3a.h:270-273,
 * rocrand_mrg31k3p.h:227-230). */
ROCRAND_B200_FN unsigned int rocrand(rocrand_state_mrg32k3a* state)
{
    return static_cast<unsigned int>((state->next() - 1) * 1.000000048661607);
}
ROCRAND_B200_FN unsigned int rocrand(rocrand_state_mrg31k3p* state)
{
    return static_cast<unsigned int>((state->next() - 1) * 2.000000001396983862);
}
ROCRAND_B200_FN unsigned int rocrand(rocrand_state_threefry2x32_20* state)
{
    return state->next();
}
ROCRAND_B200_FN uint2 rocrand2(rocrand_state_threefry2x32_20* state)
{
    return state->next_block();
}
ROCRAND_B200_FN unsigned long long rocrand(rocrand_state_threefry2x64_20* state)
{
    return state->next();
}
ROCRAND_B200_FN ulonglong2 rocrand2(rocrand_state_threefry2x64_20* state)
{
    return state->next_block();
}
ROCRAND_B200_FN unsigned int rocrand(rocrand_state_threefry4x32_20* state)
{
    return state->next();
}
ROCRAND_B200_FN uint4 rocrand4(rocrand_state_threefry4x32_20* state)
{
    return state->next_block();
}
ROCRAND_B200_FN unsigned long long rocrand(rocrand_state_threefry4x64_20* state)
{
    return state->next();
}
ROCRAND_B200_FN ulonglong4 rocrand4(rocrand_state_threefry4x64_20* state)
{
    return state->next_block();
}
ROCRAND_B200_FN unsigned int rocrand(rocrand_state_sobol32* state)
{
    return state->next();
}
ROCRAND_B200_FN unsigned long long rocrand(rocrand_state_sobol64* state)
{
    return state->next();
}
ROCRAND_B200_FN unsigned int rocrand(rocrand_state_scrambled_sobol32* state)
{
    return state->engine.next() ^ state->scramble_constant;
}
ROCRAND_B200_FN unsigned long long rocrand(rocrand_state_scrambled_sobol64* state)
{
    return state->engine.next() ^ state->scramble_constant;
}

ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_state_philox4x32_10* state)
{
    state->skip_values(offset);
    state->refresh();
}
ROCRAND_B200_FN void skipahead_subsequence(unsigned long long subsequence, rocrand_state_philox4x32_10* state)
{
    state->skip_subsequences(subsequence);
    state->refresh();
}
/* a Philox sequence is one subsequence (rocrand_philox4x32_10.h:420-425) */
ROCRAND_B200_FN void skipahead_sequence(unsigned long long sequence, rocrand_state_philox4x32_10* state)
{
    state->skip_subsequences(sequence);
    state->refresh();
}
ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_state_xorwow* state)
{
    state->skip_values(offset);
}
ROCRAND_B200_FN void skipahead_subsequence(unsigned long long subsequence, rocrand_state_xorwow* state)
{
    state->skip_subsequences(subsequence);
}
/* an XORWOW sequence is one subsequence (rocrand_xorwow.h:300-305) */
ROCRAND_B200_FN void skipahead_sequence(unsigned long long sequence, rocrand_state_xorwow* state)
{
    state->skip_subsequences(sequence);
}
ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_state_lfsr113* state)
{
    state->skip_values(offset);
}
ROCRAND_B200_FN void skipahead_subsequence(unsigned int subsequence, rocrand_state_lfsr113* state)
{
    state->skip_subsequences(subsequence);
}
ROCRAND_B200_FN void skipahead_sequence(unsigned int sequence, rocrand_state_lfsr113* state)
{
    state->skip_subsequences(sequence);
}
ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_state_mrg32k3a* state)
{
    state->skip_values(offset);
}
ROCRAND_B200_FN void skipahead_subsequence(unsigned long long subsequence, rocrand_state_mrg32k3a* state)
{
    state->skip_subsequences(subsequence);
}
ROCRAND_B200_FN void skipahead_sequence(unsigned long long sequence, rocrand_state_mrg32k3a* state)
{
    state->skip_sequences(sequence);
}
ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_state_mrg31k3p* state)
{
    state->skip_values(offset);
}
ROCRAND_B200_FN void skipahead_subsequence(unsigned long long subsequence, rocrand_state_mrg31k3p* state)
{
    state->skip_subsequences(subsequence);
}
ROCRAND_B200_FN void skipahead_sequence(unsigned long long sequence, rocrand_state_mrg31k3p* state)
{
    state->skip_sequences(sequence);
}
template<class T, class V, int N>
ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_b200_threefry_state<T, V, N>* state)
{
    state->skip_values(offset);
    state->refresh();
}
template<class T, class V, int N>
ROCRAND_B200_FN void skipahead_subsequence(unsigned long long                          subsequence,
                                           rocrand_b200_threefry_state<T, V, N>* state)
{
    state->skip_subsequences(subsequence);
    state->refresh();
}
template<class T, class V, int N>
ROCRAND_B200_FN void skipahead_sequence(unsigned long long sequence, rocrand_b200_threefry_state<T, V, N>* state)
{
    state->skip_subsequences(sequence);
    state->refresh();
}
/* Sobol skip-ahead takes the offset as 32 bits (Sobol32) or 64 bits (Sobol64), as the
 * reference's discard does. */
ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_state_sobol32* state)
{
    state->jump(static_cast<unsigned int>(offset));
}
ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_state_sobol64* state)
{
    state->jump(offset);
}
ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_state_scrambled_sobol32* state)
{
    state->engine.jump(static_cast<unsigned int>(offset));
}
ROCRAND_B200_FN void skipahead(unsigned long long offset, rocrand_state_scrambled_sobol64* state)
{
    state->engine.jump(offset);
}

// =======================================================================================
// Uniform (rocrand_uniform.h:222-823).

ROCRAND_B200_FN float rocrand_uniform(rocrand_state_philox4x32_10* state)
{
    return rocrand_b200_detail::to_float(rocrand(state));
}
ROCRAND_B200_FN float2 rocrand_uniform2(rocrand_state_philox4x32_10* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    return float2{rocrand_b200_detail::to_float(a), rocrand_b200_detail::to_float(b)};
}
ROCRAND_B200_FN float4 rocrand_uniform4(rocrand_state_philox4x32_10* state)
{
    return rocrand_b200_detail::to_float4(rocrand4(state));
}
ROCRAND_B200_FN double rocrand_uniform_double(rocrand_state_philox4x32_10* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    return rocrand_b200_detail::to_double(a, b);
}
ROCRAND_B200_FN double2 rocrand_uniform_double2(rocrand_state_philox4x32_10* state)
{
    const uint4 v = rocrand4(state);
    return double2{rocrand_b200_detail::to_double(v.x, v.y), rocrand_b200_detail::to_double(v.z, v.w)};
}
ROCRAND_B200_FN double4 rocrand_uniform_double4(rocrand_state_philox4x32_10* state)
{
    const uint4 a = rocrand4(state);
    const uint4 b = rocrand4(state);
    return double4{rocrand_b200_detail::to_double(a.x, a.y), rocrand_b200_detail::to_double(a.z, a.w),
                   rocrand_b200_detail::to_double(b.x, b.y), rocrand_b200_detail::to_double(b.z, b.w)};
}

ROCRAND_B200_FN float rocrand_uniform(rocrand_state_xorwow* state)
{
    return rocrand_b200_detail::to_float(rocrand(state));
}
ROCRAND_B200_FN double rocrand_uniform_double(rocrand_state_xorwow* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    return rocrand_b200_detail::to_double(a, b);
}

ROCRAND_B200_FN float rocrand_uniform(rocrand_state_lfsr113* state)
{
    return rocrand_b200_detail::to_float(rocrand(state));
}
ROCRAND_B200_FN double rocrand_uniform_double(rocrand_state_lfsr113* state)
{
    return rocrand_b200_detail::to_double(rocrand(state));
}

/* MRG uniforms: raw value in [1, m1] times 1/(m1 + 1) in double; float rounds that
 * (rocrand_uniform.h:182-220). */
ROCRAND_B200_FN float rocrand_uniform(rocrand_state_mrg32k3a* state)
{
    return static_cast<float>(static_cast<double>(state->next()) * 2.3283065498378288e-10);
}
ROCRAND_B200_FN double rocrand_uniform_double(rocrand_state_mrg32k3a* state)
{
    return static_cast<double>(state->next()) * 2.3283065498378288e-10;
}
ROCRAND_B200_FN float rocrand_uniform(rocrand_state_mrg31k3p* state)
{
    return static_cast<float>(static_cast<double>(state->next()) * 4.656612875245796923e-10);
}
ROCRAND_B200_FN double rocrand_uniform_double(rocrand_state_mrg31k3p* state)
{
    return static_cast<double>(state->next()) * 4.656612875245796923e-10;
}

template<class T, class V, int N>
ROCRAND_B200_FN float rocrand_uniform(rocrand_b200_threefry_state<T, V, N>* state)
{
    return rocrand_b200_detail::to_float(rocrand(state));
}
template<class T, class V, int N>
ROCRAND_B200_FN double rocrand_uniform_double(rocrand_b200_threefry_state<T, V, N>* state)
{
    return rocrand_b200_detail::to_double(rocrand(state));
}

#define ROCRAND_B200_QUASI_UNIFORM(S)                                      \
    ROCRAND_B200_FN float rocrand_uniform(S* state)                        \
    {                                                                      \
        return rocrand_b200_detail::to_float(rocrand(state));              \
    }                                                                      \
    ROCRAND_B200_FN double rocrand_uniform_double(S* state)                \
    {                                                                      \
        return rocrand_b200_detail::to_double(rocrand(state));             \
    }
ROCRAND_B200_QUASI_UNIFORM(rocrand_state_sobol32)
ROCRAND_B200_QUASI_UNIFORM(rocrand_state_sobol64)
ROCRAND_B200_QUASI_UNIFORM(rocrand_state_scrambled_sobol32)
ROCRAND_B200_QUASI_UNIFORM(rocrand_state_scrambled_sobol64)
#undef ROCRAND_B200_QUASI_UNIFORM

// =======================================================================================
// Normal (rocrand_normal.h:360-1450) and log-normal (rocrand_log_normal.h).

namespace rocrand_b200_detail
{

// MRG Box-Muller: the engine's own float uniforms (rocrand_normal.h:139-172); the double
// variant widens the float uniforms.
template<class S>
ROCRAND_B200_FN float2 mrg_box_muller(unsigned int x, unsigned int y)
{
    float2 r;
    float  u = static_cast<float>(static_cast<double>(x) * S::kNorm);
    float  v = static_cast<float>(static_cast<double>(y) * S::kNorm) * ROCRAND_2PI;
    float  s = sqrtf(-2.0f * logf(u));
#if defined(__CUDA_ARCH__)
    __sincosf(v, &r.x, &r.y);
    r.x *= s;
    r.y *= s;
#else
    r.x = sinf(v) * s;
    r.y = cosf(v) * s;
#endif
    return r;
}
template<class S>
ROCRAND_B200_FN double2 mrg_box_muller_double(unsigned int x, unsigned int y)
{
    double2 r;
    double  u = static_cast<float>(static_cast<double>(x) * S::kNorm);
    double  v = static_cast<float>(static_cast<double>(y) * S::kNorm) * 2.0;
    double  s = sqrt(-2.0 * log(u));
#if defined(__CUDA_ARCH__)
    sincospi(v, &r.x, &r.y);
    r.x *= s;
    r.y *= s;
#else
    r.x = sin(v * ROCRAND_PI_DOUBLE) * s;
    r.y = cos(v * ROCRAND_PI_DOUBLE) * s;
#endif
    return r;
}
struct Mrg32k3aNorm
{
    static constexpr double kNorm = 2.3283065498378288e-10;
};
struct Mrg31k3pNorm
{
    static constexpr double kNorm = 4.656612875245796923e-10;
};

} // namespace rocrand_b200_detail

// ---- Philox: Box-Muller on pairs of values, one cached ----
ROCRAND_B200_FN float rocrand_normal(rocrand_state_philox4x32_10* state)
{
    if(rocrand_b200_detail::bm_has_float(state))
        return rocrand_b200_detail::bm_take_float(state);
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const float2       r = rocrand_b200_detail::box_muller(a, b);
    rocrand_b200_detail::bm_keep_float(state, r.y);
    return r.x;
}
ROCRAND_B200_FN float2 rocrand_normal2(rocrand_state_philox4x32_10* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    return rocrand_b200_detail::box_muller(a, b);
}
ROCRAND_B200_FN float4 rocrand_normal4(rocrand_state_philox4x32_10* state)
{
    return rocrand_b200_detail::box_muller4(rocrand4(state));
}
ROCRAND_B200_FN double rocrand_normal_double(rocrand_state_philox4x32_10* state)
{
    if(rocrand_b200_detail::bm_has_double(state))
        return rocrand_b200_detail::bm_take_double(state);
    const double2 r = rocrand_b200_detail::box_muller_double(rocrand4(state));
    rocrand_b200_detail::bm_keep_double(state, r.y);
    return r.x;
}
ROCRAND_B200_FN double2 rocrand_normal_double2(rocrand_state_philox4x32_10* state)
{
    return rocrand_b200_detail::box_muller_double(rocrand4(state));
}
ROCRAND_B200_FN double4 rocrand_normal_double4(rocrand_state_philox4x32_10* state)
{
    const double2 r1 = rocrand_b200_detail::box_muller_double(rocrand4(state));
    const double2 r2 = rocrand_b200_detail::box_muller_double(rocrand4(state));
    return double4{r1.x, r1.y, r2.x, r2.y};
}
ROCRAND_B200_FN float rocrand_log_normal(rocrand_state_philox4x32_10* state, float mean, float stddev)
{
    if(rocrand_b200_detail::bm_has_float(state))
        return expf(mean + (stddev * rocrand_b200_detail::bm_take_float(state)));
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const float2       r = rocrand_b200_detail::box_muller(a, b);
    rocrand_b200_detail::bm_keep_float(state, r.y);
    return expf(mean + (stddev * r.x));
}
ROCRAND_B200_FN float2 rocrand_log_normal2(rocrand_state_philox4x32_10* state, float mean, float stddev)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const float2       r = rocrand_b200_detail::box_muller(a, b);
    return float2{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y))};
}
ROCRAND_B200_FN float4 rocrand_log_normal4(rocrand_state_philox4x32_10* state, float mean, float stddev)
{
    const float4 r = rocrand_b200_detail::box_muller4(rocrand4(state));
    return float4{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y)), expf(mean + (stddev * r.z)),
                  expf(mean + (stddev * r.w))};
}
ROCRAND_B200_FN double rocrand_log_normal_double(rocrand_state_philox4x32_10* state, double mean, double stddev)
{
    if(rocrand_b200_detail::bm_has_double(state))
        return exp(mean + (stddev * rocrand_b200_detail::bm_take_double(state)));
    const double2 r = rocrand_b200_detail::box_muller_double(rocrand4(state));
    rocrand_b200_detail::bm_keep_double(state, r.y);
    return exp(mean + r.x * stddev);
}
ROCRAND_B200_FN double2 rocrand_log_normal_double2(rocrand_state_philox4x32_10* state, double mean, double stddev)
{
    const double2 r = rocrand_b200_detail::box_muller_double(rocrand4(state));
    return double2{exp(mean + (stddev * r.x)), exp(mean + (stddev * r.y))};
}
ROCRAND_B200_FN double4 rocrand_log_normal_double4(rocrand_state_philox4x32_10* state, double mean, double stddev)
{
    const double2 r1 = rocrand_b200_detail::box_muller_double(rocrand4(state));
    const double2 r2 = rocrand_b200_detail::box_muller_double(rocrand4(state));
    return double4{exp(mean + (stddev * r1.x)), exp(mean + (stddev * r1.y)), exp(mean + (stddev * r2.x)),
                   exp(mean + (stddev * r2.y))};
}

// ---- XORWOW: Box-Muller on pairs (fp32) and quadruples (fp64) of values, one cached ----
ROCRAND_B200_FN float rocrand_normal(rocrand_state_xorwow* state)
{
    if(rocrand_b200_detail::bm_has_float(state))
        return rocrand_b200_detail::bm_take_float(state);
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const float2       r = rocrand_b200_detail::box_muller(a, b);
    rocrand_b200_detail::bm_keep_float(state, r.y);
    return r.x;
}
ROCRAND_B200_FN float2 rocrand_normal2(rocrand_state_xorwow* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    return rocrand_b200_detail::box_muller(a, b);
}
ROCRAND_B200_FN uint4 rocrand_b200_xorwow_quad(rocrand_state_xorwow* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const unsigned int c = rocrand(state);
    const unsigned int d = rocrand(state);
    return make_uint4(a, b, c, d);
}
ROCRAND_B200_FN double rocrand_normal_double(rocrand_state_xorwow* state)
{
    if(rocrand_b200_detail::bm_has_double(state))
        return rocrand_b200_detail::bm_take_double(state);
    const double2 r = rocrand_b200_detail::box_muller_double(rocrand_b200_xorwow_quad(state));
    rocrand_b200_detail::bm_keep_double(state, r.y);
    return r.x;
}
ROCRAND_B200_FN double2 rocrand_normal_double2(rocrand_state_xorwow* state)
{
    return rocrand_b200_detail::box_muller_double(rocrand_b200_xorwow_quad(state));
}
ROCRAND_B200_FN float rocrand_log_normal(rocrand_state_xorwow* state, float mean, float stddev)
{
    if(rocrand_b200_detail::bm_has_float(state))
        return expf(mean + (stddev * rocrand_b200_detail::bm_take_float(state)));
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const float2       r = rocrand_b200_detail::box_muller(a, b);
    rocrand_b200_detail::bm_keep_float(state, r.y);
    return expf(mean + (stddev * r.x));
}
ROCRAND_B200_FN float2 rocrand_log_normal2(rocrand_state_xorwow* state, float mean, float stddev)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const float2       r = rocrand_b200_detail::box_muller(a, b);
    return float2{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y))};
}
ROCRAND_B200_FN double rocrand_log_normal_double(rocrand_state_xorwow* state, double mean, double stddev)
{
    if(rocrand_b200_detail::bm_has_double(state))
        return exp(mean + (stddev * rocrand_b200_detail::bm_take_double(state)));
    const double2 r = rocrand_b200_detail::box_muller_double(rocrand_b200_xorwow_quad(state));
    rocrand_b200_detail::bm_keep_double(state, r.y);
    return exp(mean + (stddev * r.x));
}
ROCRAND_B200_FN double2 rocrand_log_normal_double2(rocrand_state_xorwow* state, double mean, double stddev)
{
    const double2 r = rocrand_b200_detail::box_muller_double(rocrand_b200_xorwow_quad(state));
    return double2{exp(mean + (stddev * r.x)), exp(mean + (stddev * r.y))};
}

// ---- LFSR113: the inverse-erf normal for single values, Box-Muller for pairs, no cache ----
ROCRAND_B200_FN float rocrand_normal(rocrand_state_lfsr113* state)
{
    return rocrand_b200_detail::normal_inv(rocrand(state));
}
ROCRAND_B200_FN float2 rocrand_normal2(rocrand_state_lfsr113* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    return rocrand_b200_detail::box_muller(a, b);
}
ROCRAND_B200_FN double rocrand_normal_double(rocrand_state_lfsr113* state)
{
    return rocrand_b200_detail::normal_inv_double(rocrand(state));
}
ROCRAND_B200_FN uint4 rocrand_b200_lfsr113_quad(rocrand_state_lfsr113* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const unsigned int c = rocrand(state);
    const unsigned int d = rocrand(state);
    return make_uint4(a, b, c, d);
}
ROCRAND_B200_FN double2 rocrand_normal_double2(rocrand_state_lfsr113* state)
{
    return rocrand_b200_detail::box_muller_double(rocrand_b200_lfsr113_quad(state));
}
ROCRAND_B200_FN float rocrand_log_normal(rocrand_state_lfsr113* state, float mean, float stddev)
{
    float r = rocrand_b200_detail::normal_inv(rocrand(state));
    return expf(mean + (stddev * r));
}
ROCRAND_B200_FN float2 rocrand_log_normal2(rocrand_state_lfsr113* state, float mean, float stddev)
{
    const float2 r = rocrand_normal2(state);
    return float2{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y))};
}
ROCRAND_B200_FN double rocrand_log_normal_double(rocrand_state_lfsr113* state, double mean, double stddev)
{
    double r = rocrand_b200_detail::normal_inv_double(rocrand(state));
    return exp(mean + (stddev * r));
}
ROCRAND_B200_FN double2 rocrand_log_normal_double2(rocrand_state_lfsr113* state, double mean, double stddev)
{
    const double2 r = rocrand_b200_detail::box_muller_double(rocrand_b200_lfsr113_quad(state));
    return double2{exp(mean + (stddev * r.x)), exp(mean + (stddev * r.y))};
}

// ---- MRG: Box-Muller on the engine's own uniforms, one cached ----
#define ROCRAND_B200_MRG_NORMAL(S, NORM)                                                                   \
    ROCRAND_B200_FN float rocrand_normal(S* state)                                                         \
    {                                                                                                      \
        if(rocrand_b200_detail::bm_has_float(state))                                                       \
            return rocrand_b200_detail::bm_take_float(state);                                              \
        const unsigned int a = state->next();                                                              \
        const unsigned int b = state->next();                                                              \
        const float2       r = rocrand_b200_detail::mrg_box_muller<NORM>(a, b);                            \
        rocrand_b200_detail::bm_keep_float(state, r.y);                                                    \
        return r.x;                                                                                        \
    }                                                                                                      \
    ROCRAND_B200_FN float2 rocrand_normal2(S* state)                                                       \
    {                                                                                                      \
        const unsigned int a = state->next();                                                              \
        const unsigned int b = state->next();                                                              \
        return rocrand_b200_detail::mrg_box_muller<NORM>(a, b);                                            \
    }                                                                                                      \
    ROCRAND_B200_FN double rocrand_normal_double(S* state)                                                 \
    {                                                                                                      \
        if(rocrand_b200_detail::bm_has_double(state))                                                      \
            return rocrand_b200_detail::bm_take_double(state);                                             \
        const unsigned int a = state->next();                                                              \
        const unsigned int b = state->next();                                                              \
        const double2      r = rocrand_b200_detail::mrg_box_muller_double<NORM>(a, b);                     \
        rocrand_b200_detail::bm_keep_double(state, r.y);                                                   \
        return r.x;                                                                                        \
    }                                                                                                      \
    ROCRAND_B200_FN double2 rocrand_normal_double2(S* state)                                               \
    {                                                                                                      \
        const unsigned int a = state->next();                                                              \
        const unsigned int b = state->next();                                                              \
        return rocrand_b200_detail::mrg_box_muller_double<NORM>(a, b);                                     \
    }                                                                                                      \
    ROCRAND_B200_FN float rocrand_log_normal(S* state, float mean, float stddev)                           \
    {                                                                                                      \
        if(rocrand_b200_detail::bm_has_float(state))                                                       \
            return expf(mean + (stddev * rocrand_b200_detail::bm_take_float(state)));                      \
        const unsigned int a = state->next();                                                              \
        const unsigned int b = state->next();                                                              \
        const float2       r = rocrand_b200_detail::mrg_box_muller<NORM>(a, b);                            \
        rocrand_b200_detail::bm_keep_float(state, r.y);                                                    \
        return expf(mean + (stddev * r.x));                                                                \
    }                                                                                                      \
    ROCRAND_B200_FN float2 rocrand_log_normal2(S* state, float mean, float stddev)                         \
    {                                                                                                      \
        const unsigned int a = state->next();                                                              \
        const unsigned int b = state->next();                                                              \
        const float2       r = rocrand_b200_detail::mrg_box_muller<NORM>(a, b);                            \
        return float2{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y))};                           \
    }                                                                                                      \
    ROCRAND_B200_FN double rocrand_log_normal_double(S* state, double mean, double stddev)                 \
    {                                                                                                      \
        if(rocrand_b200_detail::bm_has_double(state))                                                      \
            return exp(mean + (stddev * rocrand_b200_detail::bm_take_double(state)));                     \
        const unsigned int a = state->next();                                                              \
        const unsigned int b = state->next();                                                              \
        const double2      r = rocrand_b200_detail::mrg_box_muller_double<NORM>(a, b);                     \
        rocrand_b200_detail::bm_keep_double(state, r.y);                                                   \
        return exp(mean + r.x * stddev);                                                                   \
    }                                                                                                      \
    ROCRAND_B200_FN double2 rocrand_log_normal_double2(S* state, double mean, double stddev)               \
    {                                                                                                      \
        const unsigned int a = state->next();                                                              \
        const unsigned int b = state->next();                                                              \
        const double2      r = rocrand_b200_detail::mrg_box_muller_double<NORM>(a, b);                     \
        return double2{exp(mean + (stddev * r.x)), exp(mean + (stddev * r.y))};                            \
    }
ROCRAND_B200_MRG_NORMAL(rocrand_state_mrg32k3a, rocrand_b200_detail::Mrg32k3aNorm)
ROCRAND_B200_MRG_NORMAL(rocrand_state_mrg31k3p, rocrand_b200_detail::Mrg31k3pNorm)
#undef ROCRAND_B200_MRG_NORMAL

// ---- ThreeFry: the inverse-erf normal for single values, Box-Muller for pairs ----
/* rocrand_normal / rocrand_normal_double of every ThreeFry state: one word through the
 * inverse-erf transform (32-bit words as uint, 64-bit ones as ulonglong). */
template<class T, class V, int N>
ROCRAND_B200_FN float rocrand_normal(rocrand_b200_threefry_state<T, V, N>* state)
{
    return rocrand_b200_detail::normal_inv(rocrand(state));
}
template<class T, class V, int N>
ROCRAND_B200_FN double rocrand_normal_double(rocrand_b200_threefry_state<T, V, N>* state)
{
    return rocrand_b200_detail::normal_inv_double(rocrand(state));
}
/* log-normal single values take double mean / stddev and round the argument of expf to
 * float (rocrand_log_normal.h, ThreeFry overloads) */
template<class T, class V, int N>
ROCRAND_B200_FN float rocrand_log_normal(rocrand_b200_threefry_state<T, V, N>* state, double mean,
                                         double stddev)
{
    float r = rocrand_b200_detail::normal_inv(rocrand(state));
    return expf(mean + (stddev * r));
}
template<class T, class V, int N>
ROCRAND_B200_FN double rocrand_log_normal_double(rocrand_b200_threefry_state<T, V, N>* state, double mean,
                                                 double stddev)
{
    double r = rocrand_b200_detail::normal_inv_double(rocrand(state));
    return exp(mean + (stddev * r));
}

// pairs: each state has its own input words (rocrand_normal.h:1110-1450)
ROCRAND_B200_FN float2 rocrand_normal2(rocrand_state_threefry2x32_20* state)
{
    const uint2 v = rocrand2(state);
    return rocrand_b200_detail::box_muller(v.x, v.y);
}
ROCRAND_B200_FN float2 rocrand_normal2(rocrand_state_threefry2x64_20* state)
{
    return rocrand_b200_detail::box_muller(rocrand(state));
}
ROCRAND_B200_FN float2 rocrand_normal2(rocrand_state_threefry4x32_20* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    return rocrand_b200_detail::box_muller(a, b);
}
/* two 64-bit words reach the 32-bit Box-Muller as their low halves */
ROCRAND_B200_FN float2 rocrand_normal2(rocrand_state_threefry4x64_20* state)
{
    const unsigned long long a = rocrand(state);
    const unsigned long long b = rocrand(state);
    return rocrand_b200_detail::box_muller(static_cast<unsigned int>(a), static_cast<unsigned int>(b));
}
ROCRAND_B200_FN double2 rocrand_normal_double2(rocrand_state_threefry2x32_20* state)
{
    const uint2 a = rocrand2(state);
    const uint2 b = rocrand2(state);
    return rocrand_b200_detail::box_muller_double(make_uint4(a.x, a.y, b.x, b.y));
}
ROCRAND_B200_FN double2 rocrand_normal_double2(rocrand_state_threefry2x64_20* state)
{
    return rocrand_b200_detail::box_muller_double(rocrand2(state));
}
ROCRAND_B200_FN double2 rocrand_normal_double2(rocrand_state_threefry4x32_20* state)
{
    return rocrand_b200_detail::box_muller_double(rocrand4(state));
}
ROCRAND_B200_FN double2 rocrand_normal_double2(rocrand_state_threefry4x64_20* state)
{
    const unsigned long long a = rocrand(state);
    const unsigned long long b = rocrand(state);
    return rocrand_b200_detail::box_muller_double(ulonglong2{a, b});
}
ROCRAND_B200_FN float2 rocrand_log_normal2(rocrand_state_threefry2x32_20* state, float mean, float stddev)
{
    const float2 r = rocrand_normal2(state);
    return float2{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y))};
}
/* log-normal pairs of the 64-bit states take two words' low halves (unlike rocrand_normal2
 * of ThreeFry2x64, which splits one word) */
ROCRAND_B200_FN float2 rocrand_log_normal2(rocrand_state_threefry2x64_20* state, float mean, float stddev)
{
    const unsigned long long a = rocrand(state);
    const unsigned long long b = rocrand(state);
    const float2 r = rocrand_b200_detail::box_muller(static_cast<unsigned int>(a), static_cast<unsigned int>(b));
    return float2{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y))};
}
ROCRAND_B200_FN float2 rocrand_log_normal2(rocrand_state_threefry4x32_20* state, float mean, float stddev)
{
    const float2 r = rocrand_normal2(state);
    return float2{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y))};
}
ROCRAND_B200_FN float2 rocrand_log_normal2(rocrand_state_threefry4x64_20* state, float mean, float stddev)
{
    const float2 r = rocrand_normal2(state);
    return float2{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y))};
}
ROCRAND_B200_FN double2 rocrand_log_normal_double2(rocrand_state_threefry2x32_20* state, double mean, double stddev)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const unsigned int c = rocrand(state);
    const unsigned int d = rocrand(state);
    const double2      r = rocrand_b200_detail::box_muller_double(make_uint4(a, b, c, d));
    return double2{exp(mean + (stddev * r.x)), exp(mean + (stddev * r.y))};
}
ROCRAND_B200_FN double2 rocrand_log_normal_double2(rocrand_state_threefry2x64_20* state, double mean, double stddev)
{
    const double2 r = rocrand_normal_double2(state);
    return double2{exp(mean + (stddev * r.x)), exp(mean + (stddev * r.y))};
}
ROCRAND_B200_FN double2 rocrand_log_normal_double2(rocrand_state_threefry4x32_20* state, double mean, double stddev)
{
    const double2 r = rocrand_normal_double2(state);
    return double2{exp(mean + (stddev * r.x)), exp(mean + (stddev * r.y))};
}
ROCRAND_B200_FN double2 rocrand_log_normal_double2(rocrand_state_threefry4x64_20* state, double mean, double stddev)
{
    const double2 r = rocrand_normal_double2(state);
    return double2{exp(mean + (stddev * r.x)), exp(mean + (stddev * r.y))};
}

// ---- Sobol: the inverse-erf normal of each point ----
#define ROCRAND_B200_QUASI_NORMAL(S)                                                          \
    ROCRAND_B200_FN float rocrand_normal(S* state)                                            \
    {                                                                                         \
        return rocrand_b200_detail::normal_inv(rocrand(state));                               \
    }                                                                                         \
    ROCRAND_B200_FN double rocrand_normal_double(S* state)                                    \
    {                                                                                         \
        return rocrand_b200_detail::normal_inv_double(rocrand(state));                        \
    }                                                                                         \
    ROCRAND_B200_FN float rocrand_log_normal(S* state, float mean, float stddev)              \
    {                                                                                         \
        float r = rocrand_b200_detail::normal_inv(rocrand(state));                            \
        return expf(mean + (stddev * r));                                                     \
    }                                                                                         \
    ROCRAND_B200_FN double rocrand_log_normal_double(S* state, double mean, double stddev)    \
    {                                                                                         \
        double r = rocrand_b200_detail::normal_inv_double(rocrand(state));                    \
        return exp(mean + (stddev * r));                                                      \
    }
ROCRAND_B200_QUASI_NORMAL(rocrand_state_sobol32)
ROCRAND_B200_QUASI_NORMAL(rocrand_state_sobol64)
ROCRAND_B200_QUASI_NORMAL(rocrand_state_scrambled_sobol32)
ROCRAND_B200_QUASI_NORMAL(rocrand_state_scrambled_sobol64)
#undef ROCRAND_B200_QUASI_NORMAL

// =======================================================================================
// Poisson (rocrand_poisson.h:205-516) and discrete (rocrand_discrete.h:127-496).

ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_state_philox4x32_10* state, double lambda)
{
    return rocrand_b200_detail::poisson_rejection(state, lambda);
}
ROCRAND_B200_FN uint4 rocrand_poisson4(rocrand_state_philox4x32_10* state, double lambda)
{
    const unsigned int a = rocrand_b200_detail::poisson_rejection(state, lambda);
    const unsigned int b = rocrand_b200_detail::poisson_rejection(state, lambda);
    const unsigned int c = rocrand_b200_detail::poisson_rejection(state, lambda);
    const unsigned int d = rocrand_b200_detail::poisson_rejection(state, lambda);
    return uint4{a, b, c, d};
}
ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_state_xorwow* state, double lambda)
{
    return rocrand_b200_detail::poisson_rejection(state, lambda);
}
ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_state_lfsr113* state, double lambda)
{
    return rocrand_b200_detail::poisson_inversion(state, lambda);
}
ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_state_mrg32k3a* state, double lambda)
{
    return rocrand_b200_detail::poisson_rejection(state, lambda);
}
ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_state_mrg31k3p* state, double lambda)
{
    return rocrand_b200_detail::poisson_rejection(state, lambda);
}
template<class T, class V, int N>
ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_b200_threefry_state<T, V, N>* state, double lambda)
{
    return rocrand_b200_detail::poisson_inversion(state, lambda);
}
ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_state_sobol32* state, double lambda)
{
    return rocrand_b200_detail::poisson_inversion(state, lambda);
}
ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_state_sobol64* state, double lambda)
{
    return rocrand_b200_detail::poisson_inversion(state, lambda);
}
ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_state_scrambled_sobol32* state, double lambda)
{
    return rocrand_b200_detail::poisson_inversion(state, lambda);
}
ROCRAND_B200_FN unsigned int rocrand_poisson(rocrand_state_scrambled_sobol64* state, double lambda)
{
    return rocrand_b200_detail::poisson_inversion(state, lambda);
}

ROCRAND_B200_FN unsigned int rocrand_discrete(rocrand_state_philox4x32_10*        state,
                                              const rocrand_discrete_distribution discrete_distribution)
{
    return rocrand_b200_detail::alias_pick(rocrand(state), *discrete_distribution);
}
ROCRAND_B200_FN uint4 rocrand_discrete4(rocrand_state_philox4x32_10*        state,
                                        const rocrand_discrete_distribution discrete_distribution)
{
    const uint4 v = rocrand4(state);
    return uint4{rocrand_b200_detail::alias_pick(v.x, *discrete_distribution),
                 rocrand_b200_detail::alias_pick(v.y, *discrete_distribution),
                 rocrand_b200_detail::alias_pick(v.z, *discrete_distribution),
                 rocrand_b200_detail::alias_pick(v.w, *discrete_distribution)};
}
ROCRAND_B200_FN unsigned int rocrand_discrete(rocrand_state_xorwow*               state,
                                              const rocrand_discrete_distribution discrete_distribution)
{
    return rocrand_b200_detail::alias_pick(rocrand(state), *discrete_distribution);
}
ROCRAND_B200_FN unsigned int rocrand_discrete(rocrand_state_lfsr113*              state,
                                              const rocrand_discrete_distribution discrete_distribution)
{
    return rocrand_b200_detail::alias_pick(rocrand(state), *discrete_distribution);
}
ROCRAND_B200_FN unsigned int rocrand_discrete(rocrand_state_mrg32k3a*             state,
                                              const rocrand_discrete_distribution discrete_distribution)
{
    return rocrand_b200_detail::alias_pick(rocrand(state), *discrete_distribution);
}
ROCRAND_B200_FN unsigned int rocrand_discrete(rocrand_state_mrg31k3p*             state,
                                              const rocrand_discrete_distribution discrete_distribution)
{
    return rocrand_b200_detail::alias_pick(rocrand(state), *discrete_distribution);
}
template<class T, class V, int N>
ROCRAND_B200_FN unsigned int rocrand_discrete(rocrand_b200_threefry_state<T, V, N>* state,
                                              const rocrand_discrete_distribution          discrete_distribution)
{
    return rocrand_b200_detail::alias_pick(rocrand(state), *discrete_distribution);
}
#define ROCRAND_B200_QUASI_DISCRETE(S)                                                                \
    ROCRAND_B200_FN unsigned int rocrand_discrete(S* state,                                           \
                                                  const rocrand_discrete_distribution discrete_distribution) \
    {                                                                                                 \
        return rocrand_b200_detail::cdf_pick(rocrand(state), *discrete_distribution);                 \
    }
ROCRAND_B200_QUASI_DISCRETE(rocrand_state_sobol32)
ROCRAND_B200_QUASI_DISCRETE(rocrand_state_sobol64)
ROCRAND_B200_QUASI_DISCRETE(rocrand_state_scrambled_sobol32)
ROCRAND_B200_QUASI_DISCRETE(rocrand_state_scrambled_sobol64)
#undef ROCRAND_B200_QUASI_DISCRETE

// =======================================================================================
// MTGP32: every function is called by all threads of the block together.

#if defined(__CUDACC__)
__device__ __forceinline__ unsigned int rocrand(rocrand_state_mtgp32* state)
{
    return state->next();
}
__device__ __forceinline__ float rocrand_uniform(rocrand_state_mtgp32* state)
{
    return rocrand_b200_detail::to_float(rocrand(state));
}
__device__ __forceinline__ double rocrand_uniform_double(rocrand_state_mtgp32* state)
{
    return rocrand_b200_detail::to_double(rocrand(state));
}
__device__ __forceinline__ float rocrand_normal(rocrand_state_mtgp32* state)
{
    return rocrand_b200_detail::normal_inv(rocrand(state));
}
__device__ __forceinline__ float2 rocrand_normal2(rocrand_state_mtgp32* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    return rocrand_b200_detail::box_muller(a, b);
}
__device__ __forceinline__ double rocrand_normal_double(rocrand_state_mtgp32* state)
{
    return rocrand_b200_detail::normal_inv_double(rocrand(state));
}
__device__ __forceinline__ uint4 rocrand_b200_mtgp32_quad(rocrand_state_mtgp32* state)
{
    const unsigned int a = rocrand(state);
    const unsigned int b = rocrand(state);
    const unsigned int c = rocrand(state);
    const unsigned int d = rocrand(state);
    return make_uint4(a, b, c, d);
}
__device__ __forceinline__ double2 rocrand_normal_double2(rocrand_state_mtgp32* state)
{
    return rocrand_b200_detail::box_muller_double(rocrand_b200_mtgp32_quad(state));
}
__device__ __forceinline__ float rocrand_log_normal(rocrand_state_mtgp32* state, float mean, float stddev)
{
    float r = rocrand_b200_detail::normal_inv(rocrand(state));
    return expf(mean + (stddev * r));
}
__device__ __forceinline__ float2 rocrand_log_normal2(rocrand_state_mtgp32* state, float mean, float stddev)
{
    const float2 r = rocrand_normal2(state);
    return float2{expf(mean + (stddev * r.x)), expf(mean + (stddev * r.y))};
}
__device__ __forceinline__ double rocrand_log_normal_double(rocrand_state_mtgp32* state, double mean, double stddev)
{
    double r = rocrand_b200_detail::normal_inv_double(rocrand(state));
    return exp(mean + (stddev * r));
}
__device__ __forceinline__ double2 rocrand_log_normal_double2(rocrand_state_mtgp32* state, double mean, double stddev)
{
    const double2 r = rocrand_b200_detail::box_muller_double(rocrand_b200_mtgp32_quad(state));
    return double2{exp(mean + (stddev * r.x)), exp(mean + (stddev * r.y))};
}
__device__ __forceinline__ unsigned int rocrand_poisson(rocrand_state_mtgp32* state, double lambda)
{
    return rocrand_b200_detail::poisson_inversion(state, lambda);
}
__device__ __forceinline__ unsigned int rocrand_discrete(rocrand_state_mtgp32*               state,
                                                         const rocrand_discrete_distribution discrete_distribution)
{
    return rocrand_b200_detail::alias_pick(rocrand(state), *discrete_distribution);
}
#endif

#endif /* ROCRAND_KERNEL_H_ */
