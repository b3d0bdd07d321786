// sobol_dist.cuh -- distributions over a Sobol value and the Gray-code helpers, shared by
// the per-generator Sobol kernels (sobol.cu) and the batched fill (batch.cu).
#pragma once

#include "common.hpp"
#include "dist.cuh"
#include "logf_replay.cuh"

namespace rb200
{

// ---- distributions over a Sobol value (sobol_*_distribution, uniform.hpp:351-442,
//      normal.hpp:272-330, log_normal.hpp:296-370, poisson.hpp CDF method) ----

// rocrand_normal.h:174-194 roc_f_erfinv, every step rounded as written; the logarithm is the
// host C library's logf (logf_replay.cuh), which the outer cancellation amplifies.
RB_HD float erfinv_f(float x, const lr::Table& logf_table)
{
    const float sgn = (x < 0.0f) ? -1.0f : 1.0f;
    x               = ieee::fmul(ieee::fsub(1.0f, x), ieee::fadd(1.0f, x));
#if defined(__CUDA_ARCH__)
    const float lnx = lr::logf_host(x, logf_table);
#else
    (void)logf_table;
    const float lnx = std::log(x); // the host's own logf (the host path of host generators)
#endif
    if(isnan(lnx))
        return 1.0f;
    if(isinf(lnx))
        return 0.0f;
    const float tt1 = ieee::fadd(2.0f / (3.141592653f * 0.147f), ieee::fmul(0.5f, lnx));
    const float tt2 = ieee::fmul(1.0f / (0.147f), lnx);
    return sgn * ieee::fsqrt(ieee::fadd(-tt1, ieee::fsqrt(ieee::fsub(ieee::fmul(tt1, tt1), tt2))));
}

// normal_distribution(unsigned int) (rocrand_normal.h:228-233); a 64-bit value uses its high word.
RB_HD float sobol_normal_f(uint32_t hi32, const lr::Table& logf_table)
{
    const float p = u32_to_f32(hi32);
    return ieee::fmul(RB_SQRT2, erfinv_f(ieee::fsub(ieee::fmul(2.0f, p), 1.0f), logf_table));
}

template<class W>
RB_HD uint32_t high32(W x)
{
    return static_cast<uint32_t>(x >> (8 * sizeof(W) - 32));
}

// uniform_distribution_double over a Sobol value: 2^-32 based for 32-bit, 2^-53 for 64-bit.
template<class W>
RB_HD double sobol_u_f64(W x)
{
    if constexpr(sizeof(W) == 4)
        return u32_to_f64(x);
    else
        return ieee::dfma(ieee::ull2d(x >> 11), RB_2POW53_INV_DOUBLE, RB_2POW53_INV_DOUBLE);
}

template<class W>
RB_HD double sobol_normal_d(W x)
{
    const double p = sobol_u_f64(x);
    return ieee::dmul((double)RB_SQRT2, erfinv_d(ieee::dsub(ieee::dmul(2.0, p), 1.0)));
}

enum class SobolKind : int
{
    UINT,
    ULL,
    UCHAR,
    USHORT,
    FLOAT,
    DOUBLE,
    HALF,
    NORMAL_F,
    NORMAL_D,
    NORMAL_H,
    LOGNORMAL_F,
    LOGNORMAL_D,
    LOGNORMAL_H,
    POISSON,
    POISSON_HUGE
};

template<SobolKind K, class W>
struct SobolOut;
template<class W> struct SobolOut<SobolKind::UINT, W> { using T = uint32_t; };
template<class W> struct SobolOut<SobolKind::ULL, W> { using T = unsigned long long; };
template<class W> struct SobolOut<SobolKind::UCHAR, W> { using T = uint8_t; };
template<class W> struct SobolOut<SobolKind::USHORT, W> { using T = uint16_t; };
template<class W> struct SobolOut<SobolKind::FLOAT, W> { using T = float; };
template<class W> struct SobolOut<SobolKind::DOUBLE, W> { using T = double; };
template<class W> struct SobolOut<SobolKind::HALF, W> { using T = __half; };
template<class W> struct SobolOut<SobolKind::NORMAL_F, W> { using T = float; };
template<class W> struct SobolOut<SobolKind::NORMAL_D, W> { using T = double; };
template<class W> struct SobolOut<SobolKind::NORMAL_H, W> { using T = __half; };
template<class W> struct SobolOut<SobolKind::LOGNORMAL_F, W> { using T = float; };
template<class W> struct SobolOut<SobolKind::LOGNORMAL_D, W> { using T = double; };
template<class W> struct SobolOut<SobolKind::LOGNORMAL_H, W> { using T = __half; };
template<class W> struct SobolOut<SobolKind::POISSON, W> { using T = uint32_t; };
template<class W> struct SobolOut<SobolKind::POISSON_HUGE, W> { using T = uint32_t; };

struct SobolParams
{
    float         mean_f, std_f;
    double        mean_d, std_d;
    const double* cdf;
    uint32_t      size, offset;
    double        lambda, sqrt_lambda;
    lr::Table     logf; // fp32 normal kinds: the host-logf replay table
};

template<SobolKind K, class W>
RB_HD typename SobolOut<K, W>::T sobol_apply(W x, const SobolParams& p,
                                                                   const double* cdf)
{
    constexpr int B = 8 * sizeof(W);
    if constexpr(K == SobolKind::UINT)
        return high32(x);
    else if constexpr(K == SobolKind::ULL)
        return x;
    else if constexpr(K == SobolKind::UCHAR)
        return static_cast<uint8_t>(x >> (B - 8));
    else if constexpr(K == SobolKind::USHORT)
        return static_cast<uint16_t>(x >> (B - 16));
    else if constexpr(K == SobolKind::FLOAT)
        return u32_to_f32(high32(x));
    else if constexpr(K == SobolKind::DOUBLE)
        return sobol_u_f64(x);
    else if constexpr(K == SobolKind::HALF)
        return u16_to_f16(static_cast<uint32_t>(x >> (B - 16)) & 0xffffu);
    else if constexpr(K == SobolKind::NORMAL_F)
        return ieee::fadd(p.mean_f, ieee::fmul(sobol_normal_f(high32(x), p.logf), p.std_f));
    else if constexpr(K == SobolKind::LOGNORMAL_F)
        return ieee::expf_(ieee::fadd(p.mean_f, ieee::fmul(p.std_f, sobol_normal_f(high32(x), p.logf))));
    else if constexpr(K == SobolKind::NORMAL_D)
        return ieee::dadd(p.mean_d, ieee::dmul(sobol_normal_d(x), p.std_d));
    else if constexpr(K == SobolKind::LOGNORMAL_D)
        return ieee::exp_(ieee::dadd(p.mean_d, ieee::dmul(p.std_d, sobol_normal_d(x))));
    else if constexpr(K == SobolKind::NORMAL_H)
        return __float2half_rn(ieee::fadd(p.mean_f, ieee::fmul(sobol_normal_f(high32(x), p.logf), p.std_f)));
    else if constexpr(K == SobolKind::LOGNORMAL_H)
        return __float2half_rn(ieee::expf_(ieee::fadd(p.mean_f, ieee::fmul(p.std_f, sobol_normal_f(high32(x), p.logf)))));
    else if constexpr(K == SobolKind::POISSON)
    {
        // discrete_cdf (rocrand_discrete.h:92-115): first entry >= x, capped at the last
        double xd;
        if constexpr(sizeof(W) == 4)
            xd = ieee::dmul(ieee::u2d(x), RB_2POW32_INV_DOUBLE);
        else
            xd = ieee::dmul(ieee::ull2d(x), 5.4210108624275221700372640043497e-20);
        uint32_t lo = 0, hi = p.size - 1;
        while(lo != hi)
        {
            const uint32_t c = (lo + hi) / 2;
            if(xd > cdf[c])
                lo = c + 1;
            else
                hi = c;
        }
        return p.offset + lo;
    }
    else
    {
        static_assert(K == SobolKind::POISSON_HUGE, "kind");
        const double nd = sobol_normal_d(x);
        return (uint32_t)(long long)round(ieee::dadd(ieee::dmul(p.sqrt_lambda, nd), p.lambda));
    }
}

// Index of the rightmost zero bit of x; an all-ones x (the 32-bit point counter at its
// last value) gives 0, as the reference's device engine does (rocrand_sobol32.h:161-166),
// which also keeps the table index in range.
template<class W>
RB_HD uint32_t rzb(W x)
{
    int z;
    if constexpr(sizeof(W) == 4)
    {
#if defined(__CUDA_ARCH__)
        z = __ffs(~x);
#else
        z = __builtin_ffs(static_cast<int>(~x));
#endif
    }
    else
    {
#if defined(__CUDA_ARCH__)
        z = __ffsll(static_cast<long long>(~x));
#else
        z = __builtin_ffsll(static_cast<long long>(~x));
#endif
    }
    return z ? static_cast<uint32_t>(z - 1) : 0u;
}

} // namespace rb200
