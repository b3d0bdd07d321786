// dist.cuh -- distribution functors fused into the generator kernels (sm_100a).
//
// Each functor reproduces one host functor of the reference (library/src/rng/distribution/
// *.hpp) together with the scalar conversion it calls in the *host* branch of
// library/include/rocrand/rocrand_{uniform,normal,discrete}.h, because parity is defined
// against the reference's host generators.  Every rounding step is written with an
// explicit _rn intrinsic: a product is fused into an FMA only where it is exact (scaling
// by a power of two), so the device rounds exactly where the x86-64 host does.
// fp32 transcendentals use CUDA's accurate library functions, within an ulp or two of the
// host C library, inside the stated fp32 tolerance.  The fp64 Box-Muller transforms and
// the inverse-erf normal take log/sin/cos from precise_math.cuh (correctly rounded but for
// rare near-halfway cases), so that the fp64 outputs stay within 2 ulp of the host's and
// the ill-conditioned inverse-erf formula starts from the same logarithm wherever the host
// library's is itself correctly rounded.
#pragma once

#include <type_traits>
#include "common.hpp"
#include "ieee.cuh"
#include "precise_math.cuh"

#include <cuda_fp16.h>

#include <cstdint>

namespace rb200
{

// Constants of rocrand_common.h:24-36, spelled as the reference spells them so that they
// round to the same binary values.
#define RB_2POW16_INV (1.5258789e-05f)
#define RB_2POW16_INV_2PI (9.58738e-05f)
#define RB_2POW32_INV (2.3283064e-10f)
#define RB_2POW32_INV_DOUBLE (2.3283064365386963e-10)
#define RB_2POW32_INV_2PI (1.46291807e-09f)
#define RB_2POW53_INV_DOUBLE (1.1102230246251565e-16)
#define RB_PI_DOUBLE (3.1415926535897932)
#define RB_SQRT2 (1.4142135f)

// ---- scalar conversions ----

// rocrand_uniform.h:61-64: 2^-32 + v * 2^-32 (exact product, one rounding).
RB_HD float u32_to_f32(uint32_t v)
{
    return ieee::ffma(ieee::u2f(v), RB_2POW32_INV, RB_2POW32_INV);
}

// rocrand_uniform.h:97-107: 53 bits from (v1, v2 >> 11), 2^-53 + v * 2^-53.
RB_HD double u32x2_to_f64(uint32_t v1, uint32_t v2)
{
    const uint64_t v = (uint64_t)v1 | ((uint64_t)(v2 >> 11) << 32);
    return ieee::dfma(ieee::ull2d(v), RB_2POW53_INV_DOUBLE, RB_2POW53_INV_DOUBLE);
}

// rocrand_uniform.h:92-95: 2^-32 + v * 2^-32 in double (exact).
RB_HD double u32_to_f64(uint32_t v)
{
    return ieee::dfma(ieee::u2d(v), RB_2POW32_INV_DOUBLE, RB_2POW32_INV_DOUBLE);
}

// rocrand_uniform.h:150-153: half of 2^-16 + v * 2^-16 (float math exact, RNE to half).
RB_HD __half u16_to_f16(uint32_t v16)
{
    return __float2half_rn(ieee::ffma((float)(v16 & 0xffffu), RB_2POW16_INV, RB_2POW16_INV));
}

// rocrand_normal.h:51-66 (host branch: sinf/cosf on the rounded angle).
RB_HD float2 box_muller_f32(uint32_t x, uint32_t y)
{
    const float u = ieee::ffma(ieee::u2f(x), RB_2POW32_INV, RB_2POW32_INV);
    const float v = ieee::fadd(RB_2POW32_INV_2PI, ieee::fmul(ieee::u2f(y), RB_2POW32_INV_2PI));
    const float s = ieee::fsqrt(ieee::fmul(-2.0f, ieee::logf_(u)));
    float       sv, cv;
    ieee::sincosf_(v, &sv, &cv);
    return make_float2(ieee::fmul(sv, s), ieee::fmul(cv, s));
}

// rocrand_normal.h:68-89 (host branch: sin/cos of w * pi rounded in double).
RB_HD double2 box_muller_f64(uint32_t x, uint32_t y, uint32_t z, uint32_t w)
{
    const uint64_t v1 = (uint64_t)x ^ ((uint64_t)y << 21);
    const double   u  = ieee::dfma(ieee::ull2d(v1), RB_2POW53_INV_DOUBLE, RB_2POW53_INV_DOUBLE);
    const uint64_t v2 = (uint64_t)z ^ ((uint64_t)w << 21);
    const double   ww = ieee::dfma(ieee::ull2d(v2), RB_2POW53_INV_DOUBLE * 2.0, RB_2POW53_INV_DOUBLE * 2.0);
    const double   s  = ieee::dsqrt(ieee::dmul(-2.0, pm::log(u)));
    const double   a  = ieee::dmul(ww, RB_PI_DOUBLE);
    double         sv, cv;
    pm::sincos(a, sv, cv);
    return make_double2(ieee::dmul(sv, s), ieee::dmul(cv, s));
}

// rocrand_normal.h:102-122, float branch used by the host build; halves of the results.
RB_HD void box_muller_f16(uint32_t v, __half r[2])
{
    const float u = ieee::ffma((float)(v & 0xffffu), RB_2POW16_INV, RB_2POW16_INV);
    const float a = ieee::fadd(RB_2POW16_INV_2PI, ieee::fmul((float)(v >> 16), RB_2POW16_INV_2PI));
    const float s = ieee::fsqrt(ieee::fmul(-2.0f, ieee::logf_(u)));
    float       sv, cv;
    ieee::sincosf_(a, &sv, &cv);
    r[0] = __float2half_rn(ieee::fmul(sv, s));
    r[1] = __float2half_rn(ieee::fmul(cv, s));
}

// rocrand_normal.h:196-220 roc_d_erfinv (host branch).
RB_HD double erfinv_d(double x)
{
    const double sgn = (x < 0.0) ? -1.0 : 1.0;
    x                = ieee::dmul(ieee::dsub(1.0, x), ieee::dadd(1.0, x));
    const double lnx = pm::log(x);
    if(isnan(lnx))
        return 1.0;
    if(isinf(lnx))
        return 0.0;
    const double tt1 = ieee::dadd(2.0 / (RB_PI_DOUBLE * 0.147), ieee::dmul(0.5, lnx));
    const double tt2 = ieee::dmul(1.0 / (0.147), lnx);
    return sgn * ieee::dsqrt(ieee::dadd(-tt1, ieee::dsqrt(ieee::dsub(ieee::dmul(tt1, tt1), tt2))));
}

// rocrand_normal.h:265-270: sqrt(2) is a float literal promoted to double.
RB_HD double normal_from_u32_f64(uint32_t x)
{
    const double p = u32_to_f64(x);
    return ieee::dmul((double)RB_SQRT2, erfinv_d(ieee::dsub(ieee::dmul(2.0, p), 1.0)));
}

// rocrand_discrete.h:33-60 discrete_alias for a 32-bit input.
RB_HD uint32_t alias_lookup(uint32_t r, uint32_t size, uint32_t offset,
                                                 const double* prob, const uint32_t* alias)
{
    const double   x   = ieee::dmul(ieee::u2d(r), RB_2POW32_INV_DOUBLE);
    const double   nx  = ieee::dmul(ieee::u2d(size), x);
    const double   fnx = floor(nx);
    const double   y   = ieee::dsub(nx, fnx);
    const uint32_t i   = ieee::d2u_rz(fnx);
    return offset + (y < prob[i] ? i : alias[i]);
}

// The same pick from packed integer entries (poisson.hpp alias_entry: threshold in the low
// 33 bits, alias above): i = (size r) >> 32, entry i when the low word of size r is below
// the threshold.  One 8-byte read, no conversion or fp64 operation.
RB_HD uint32_t alias_lookup_packed(uint32_t r, uint32_t size, uint32_t offset,
                                                        const unsigned long long* tab)
{
    const unsigned long long p  = static_cast<unsigned long long>(size) * r;
    const uint32_t           i  = static_cast<uint32_t>(p >> 32);
    const unsigned long long e  = tab[i];
    const unsigned long long lo = p & 0xffffffffull;
    return offset + (lo < (e & 0x1ffffffffull) ? i : static_cast<uint32_t>(e >> 33));
}

// poisson.hpp:80-108 poisson_distribution_huge: round(sqrt(lambda) * N + lambda).
RB_HD uint32_t poisson_huge(uint32_t r, double sqrt_lambda, double lambda)
{
    const double nd = normal_from_u32_f64(r);
    return (uint32_t)(long long)round(ieee::dadd(ieee::dmul(sqrt_lambda, nd), lambda));
}

// ---- functors: iw inputs (32-bit engine words) -> ow outputs of T ----
// Naming follows the reference entry point they serve.

struct FnUint // uniform_distribution<uint> (uniform.hpp:42-53)
{
    using T                      = uint32_t;
    static constexpr unsigned iw = 1, ow = 1;
    RB_HD void operator()(const uint32_t* in, T* out) const { out[0] = in[0]; }
};

struct FnUchar // uniform_distribution<uchar> (uniform.hpp:55-66): the word's 4 bytes
{
    using T                      = uint8_t;
    static constexpr unsigned iw = 1, ow = 4;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = (uint8_t)in[0];
        out[1] = (uint8_t)(in[0] >> 8);
        out[2] = (uint8_t)(in[0] >> 16);
        out[3] = (uint8_t)(in[0] >> 24);
    }
};

struct FnUshort // uniform_distribution<ushort> (uniform.hpp:68-79): the word's 2 halves
{
    using T                      = uint16_t;
    static constexpr unsigned iw = 1, ow = 2;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = (uint16_t)in[0];
        out[1] = (uint16_t)(in[0] >> 16);
    }
};

struct FnFloat // uniform_distribution<float> (uniform.hpp:81-91)
{
    using T                      = float;
    static constexpr unsigned iw = 1, ow = 1;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = u32_to_f32(in[0]);
    }
};

struct FnDouble // uniform_distribution<double> (uniform.hpp:93-103)
{
    using T                      = double;
    static constexpr unsigned iw = 2, ow = 1;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = u32x2_to_f64(in[0], in[1]);
    }
};

struct FnHalf // uniform_distribution<half> (uniform.hpp:105-117)
{
    using T                      = __half;
    static constexpr unsigned iw = 1, ow = 2;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = u16_to_f16(in[0] & 0xffffu);
        out[1] = u16_to_f16(in[0] >> 16);
    }
};

struct FnNormalF // normal_distribution<float, uint, 4> (normal.hpp:49-69)
{
    using T                      = float;
    static constexpr unsigned iw = 2, ow = 2;
    float                     mean, stddev;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        const float2 v = box_muller_f32(in[0], in[1]);
        out[0]         = ieee::fadd(mean, ieee::fmul(v.x, stddev));
        out[1]         = ieee::fadd(mean, ieee::fmul(v.y, stddev));
    }
};

struct FnLogNormalF // log_normal_distribution<float, uint, 4> (log_normal.hpp:51-71)
{
    using T                      = float;
    static constexpr unsigned iw = 2, ow = 2;
    float                     mean, stddev;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        const float2 v = box_muller_f32(in[0], in[1]);
        out[0]         = ieee::expf_(ieee::fadd(mean, ieee::fmul(v.x, stddev)));
        out[1]         = ieee::expf_(ieee::fadd(mean, ieee::fmul(v.y, stddev)));
    }
};

struct FnNormalD // normal_distribution<double, uint, 4> (normal.hpp:90-111)
{
    using T                      = double;
    static constexpr unsigned iw = 4, ow = 2;
    double                    mean, stddev;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        const double2 v = box_muller_f64(in[0], in[1], in[2], in[3]);
        out[0]          = ieee::dadd(mean, ieee::dmul(v.x, stddev));
        out[1]          = ieee::dadd(mean, ieee::dmul(v.y, stddev));
    }
};

struct FnLogNormalD // log_normal_distribution<double, uint, 4> (log_normal.hpp:92-113)
{
    using T                      = double;
    static constexpr unsigned iw = 4, ow = 2;
    double                    mean, stddev;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        const double2 v = box_muller_f64(in[0], in[1], in[2], in[3]);
        out[0]          = ieee::exp_(ieee::dadd(mean, ieee::dmul(v.x, stddev)));
        out[1]          = ieee::exp_(ieee::dadd(mean, ieee::dmul(v.y, stddev)));
    }
};

struct FnNormalH // normal_distribution<half, uint, 4> (normal.hpp:113-136), float branch
{
    using T                      = __half;
    static constexpr unsigned iw = 1, ow = 2;
    float                     mean, stddev; // the half parameters widened to float
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        __half r[2];
        box_muller_f16(in[0], r);
        out[0] = __float2half_rn(ieee::fadd(mean, ieee::fmul(stddev, __half2float(r[0]))));
        out[1] = __float2half_rn(ieee::fadd(mean, ieee::fmul(stddev, __half2float(r[1]))));
    }
};

struct FnLogNormalH // log_normal_distribution<half, uint, 4> (log_normal.hpp:115-139)
{
    using T                      = __half;
    static constexpr unsigned iw = 1, ow = 2;
    float                     mean, stddev;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        __half r[2];
        box_muller_f16(in[0], r);
        out[0] = __float2half_rn(ieee::expf_(ieee::fadd(mean, ieee::fmul(stddev, __half2float(r[0])))));
        out[1] = __float2half_rn(ieee::expf_(ieee::fadd(mean, ieee::fmul(stddev, __half2float(r[1])))));
    }
};

// poisson_distribution<ALIAS> (poisson.hpp:49-76).  The table is staged in shared memory
// by the kernel; prob/alias then point there.
struct FnPoisson
{
    using T                      = uint32_t;
    static constexpr unsigned iw = 1, ow = 1;
    static constexpr bool     kTable = true;
    const unsigned long long* prob;  // packed entries (alias_entry), not probabilities
    const uint32_t*           alias; // unused: the aliases are packed with the thresholds
    uint32_t                  size, offset;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = alias_lookup_packed(in[0], size, offset, prob);
    }
};

// poisson_distribution_huge (poisson.hpp:80-108), lambda > 4000.
struct FnPoissonHuge
{
    using T                      = uint32_t;
    static constexpr unsigned iw = 1, ow = 1;
    double                    sqrt_lambda, lambda;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = poisson_huge(in[0], sqrt_lambda, lambda);
    }
};

// ---- functors over 64-bit engine words (ThreeFry 2x64/4x64) ----
// uniform.hpp:119-200, normal.hpp:138-200, log_normal.hpp:138-200, and the 64-bit input
// overloads of rocrand_uniform.h / rocrand_normal.h / rocrand_discrete.h.

struct Fn64Ulonglong // uniform_distribution<ull, ull>
{
    using T                      = unsigned long long;
    static constexpr unsigned iw = 1, ow = 1;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
        out[0] = in[0];
    }
};

template<class U, unsigned N>
struct Fn64Split // uchar (ow 8), ushort (ow 4), uint (ow 2): the word's bytes in order
{
    using T                      = U;
    static constexpr unsigned iw = 1, ow = N;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
#pragma unroll
        for(unsigned k = 0; k < N; k++)
            out[k] = static_cast<U>(in[0] >> (k * 8 * sizeof(U)));
    }
};

struct Fn64Float // rocrand_uniform.h:66-69: 2^-32 + (v >> 32) * 2^-32
{
    using T                      = float;
    static constexpr unsigned iw = 1, ow = 1;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
        out[0] = u32_to_f32(static_cast<uint32_t>(in[0] >> 32));
    }
};

struct Fn64Double // rocrand_uniform.h:109-116: 2^-53 + (v >> 11) * 2^-53
{
    using T                      = double;
    static constexpr unsigned iw = 1, ow = 1;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
        out[0] = ieee::dfma(ieee::ull2d(in[0] >> 11), RB_2POW53_INV_DOUBLE, RB_2POW53_INV_DOUBLE);
    }
};

struct Fn64Half // uniform_distribution<half, ull>: four 16-bit fields
{
    using T                      = __half;
    static constexpr unsigned iw = 1, ow = 4;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
#pragma unroll
        for(unsigned k = 0; k < 4; k++)
            out[k] = u16_to_f16(static_cast<uint32_t>(in[0] >> (16 * k)) & 0xffffu);
    }
};

struct Fn64NormalF // box_muller(unsigned long long): x = low word, y = high word
{
    using T                      = float;
    static constexpr unsigned iw = 1, ow = 2;
    float                     mean, stddev;
    bool                      log_normal;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
        const float2 v = box_muller_f32(static_cast<uint32_t>(in[0]), static_cast<uint32_t>(in[0] >> 32));
        const float  a = ieee::fadd(mean, ieee::fmul(v.x, stddev));
        const float  b = ieee::fadd(mean, ieee::fmul(v.y, stddev));
        out[0]         = log_normal ? ieee::expf_(a) : a;
        out[1]         = log_normal ? ieee::expf_(b) : b;
    }
};

struct Fn64NormalD // box_muller_double(ulonglong2)
{
    using T                      = double;
    static constexpr unsigned iw = 2, ow = 2;
    double                    mean, stddev;
    bool                      log_normal;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
        const double2 v = box_muller_f64(static_cast<uint32_t>(in[0]), static_cast<uint32_t>(in[0] >> 32),
                                         static_cast<uint32_t>(in[1]), static_cast<uint32_t>(in[1] >> 32));
        const double  a = ieee::dadd(mean, ieee::dmul(v.x, stddev));
        const double  b = ieee::dadd(mean, ieee::dmul(v.y, stddev));
        out[0]          = log_normal ? ieee::exp_(a) : a;
        out[1]          = log_normal ? ieee::exp_(b) : b;
    }
};

struct Fn64NormalH // normal_distribution_half2(ull): (ushort)v and (ushort)(v >> 32)
{
    using T                      = __half;
    static constexpr unsigned iw = 1, ow = 2;
    float                     mean, stddev;
    bool                      log_normal;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
        __half         r[2];
        const uint32_t v = (static_cast<uint32_t>(in[0]) & 0xffffu)
                           | (static_cast<uint32_t>(in[0] >> 32) << 16);
        box_muller_f16(v, r);
#pragma unroll
        for(int k = 0; k < 2; k++)
        {
            const float z = ieee::fadd(mean, ieee::fmul(stddev, __half2float(r[k])));
            out[k]        = __float2half_rn(log_normal ? ieee::expf_(z) : z);
        }
    }
};

// discrete_alias(unsigned long long) (rocrand_discrete.h:75-81): x = r * 2^-64 after the
// round-to-nearest conversion of r to double.  When r rounds up to 2^64 the reference reads
// one entry past the table; here the index is clamped to the last entry instead.
struct Fn64Poisson
{
    using T                      = uint32_t;
    static constexpr unsigned iw = 1, ow = 1;
    const double*             prob;
    const uint32_t*           alias;
    uint32_t                  size, offset;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
        const double x   = ieee::dmul(ieee::ull2d(in[0]), 5.4210108624275221700372640043497e-20);
        const double nx  = ieee::dmul(ieee::u2d(size), x);
        const double fnx = floor(nx);
        const double y   = ieee::dsub(nx, fnx);
        uint32_t     i   = ieee::d2u_rz(fnx);
        i                = i < size ? i : size - 1;
        out[0]           = offset + (y < prob[i] ? i : alias[i]);
    }
};

struct Fn64PoissonHuge // normal_distribution_double(ull) then round(sqrt(l) * N + l)
{
    using T                      = uint32_t;
    static constexpr unsigned iw = 1, ow = 1;
    double                    sqrt_lambda, lambda;
    RB_HD void operator()(const unsigned long long* in, T* out) const
    {
        const double p  = ieee::dfma(ieee::ull2d(in[0] >> 11), RB_2POW53_INV_DOUBLE, RB_2POW53_INV_DOUBLE);
        const double nd = ieee::dmul((double)RB_SQRT2, erfinv_d(ieee::dsub(ieee::dmul(2.0, p), 1.0)));
        out[0]          = (uint32_t)(long long)round(ieee::dadd(ieee::dmul(sqrt_lambda, nd), lambda));
    }
};

// normal_distribution<double, uint, 2> / log_normal_distribution<double, uint, 2>
// (normal.hpp:71-88): the inverse-erf normal, one word per value; used by ThreeFry2x32.
struct FnNormalD1
{
    using T                      = double;
    static constexpr unsigned iw = 1, ow = 1;
    double                    mean, stddev;
    bool                      log_normal;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        const double z = ieee::dadd(mean, ieee::dmul(normal_from_u32_f64(in[0]), stddev));
        out[0]         = log_normal ? ieee::exp_(z) : z;
    }
};

// ---- MRG functors (uniform.hpp:224-314, normal.hpp:200-270, log_normal.hpp:200-276,
//      poisson.hpp:416-441): the raw MRG output lies in [1, m1] and is normalised by the
//      engine's own constants (rocrand_uniform.h:161-219, rocrand_normal.h:138-172). ----

struct Mrg31k3pNorm // rocrand_mrg31k3p.h:32-34
{
    static constexpr double kNorm     = 4.656612875245796923e-10;
    static constexpr double kUintNorm = 2.000000001396983862;
};
struct Mrg32k3aNorm // rocrand_mrg32k3a.h:38-39
{
    static constexpr double kNorm     = 2.3283065498378288e-10;
    static constexpr double kUintNorm = 1.000000048661607;
};

template<class N>
RB_HD uint32_t mrg_to_u32(uint32_t v) // (v - 1) * UINT_NORM, truncated
{
    return ieee::d2u_rz(ieee::dmul(ieee::u2d(v - 1u), N::kUintNorm));
}
template<class N>
RB_HD float mrg_to_f32(uint32_t v)
{
    return ieee::d2f(ieee::dmul(ieee::u2d(v), N::kNorm));
}
template<class N>
RB_HD double mrg_to_f64(uint32_t v)
{
    return ieee::dmul(ieee::u2d(v), N::kNorm);
}

template<class N, class Inner>
struct FnMrgRemap // uint/uchar/ushort/half/Poisson: remap to [0, 2^32) then the plain functor
{
    using T                      = typename Inner::T;
    static constexpr unsigned iw = 1, ow = Inner::ow;
    Inner                     inner;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        const uint32_t v = mrg_to_u32<N>(in[0]);
        inner(&v, out);
    }
};

template<class N>
struct FnMrgFloat
{
    using T                      = float;
    static constexpr unsigned iw = 1, ow = 1;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = mrg_to_f32<N>(in[0]);
    }
};

template<class N>
struct FnMrgDouble
{
    using T                      = double;
    static constexpr unsigned iw = 1, ow = 1;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = mrg_to_f64<N>(in[0]);
    }
};

template<class N>
struct FnMrgNormalF // mrg_box_muller (rocrand_normal.h:138-152)
{
    using T                      = float;
    static constexpr unsigned iw = 2, ow = 2;
    float                     mean, stddev;
    bool                      log_normal;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        const float u = mrg_to_f32<N>(in[0]);
        const float v = ieee::fmul(mrg_to_f32<N>(in[1]), 6.2831855f);
        const float s = ieee::fsqrt(ieee::fmul(-2.0f, ieee::logf_(u)));
        float       sv, cv;
        ieee::sincosf_(v, &sv, &cv);
        const float a = ieee::fadd(mean, ieee::fmul(ieee::fmul(sv, s), stddev));
        const float b = ieee::fadd(mean, ieee::fmul(ieee::fmul(cv, s), stddev));
        out[0]        = log_normal ? ieee::expf_(a) : a;
        out[1]        = log_normal ? ieee::expf_(b) : b;
    }
};

template<class N>
struct FnMrgNormalD // mrg_box_muller_double (rocrand_normal.h:154-172): float uniforms widened
{
    using T                      = double;
    static constexpr unsigned iw = 2, ow = 2;
    double                    mean, stddev;
    bool                      log_normal;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        const double u = (double)mrg_to_f32<N>(in[0]);
        const double v = (double)mrg_to_f32<N>(in[1]) * 2.0;
        const double s = ieee::dsqrt(ieee::dmul(-2.0, pm::log(u)));
        double       sv, cv;
        pm::sincos(ieee::dmul(v, RB_PI_DOUBLE), sv, cv);
        const double a = ieee::dadd(mean, ieee::dmul(ieee::dmul(sv, s), stddev));
        const double b = ieee::dadd(mean, ieee::dmul(ieee::dmul(cv, s), stddev));
        out[0]         = log_normal ? ieee::exp_(a) : a;
        out[1]         = log_normal ? ieee::exp_(b) : b;
    }
};

template<class N>
struct FnMrgPoissonHuge
{
    using T                      = uint32_t;
    static constexpr unsigned iw = 1, ow = 1;
    double                    sqrt_lambda, lambda;
    RB_HD void operator()(const uint32_t* in, T* out) const
    {
        out[0] = poisson_huge(mrg_to_u32<N>(in[0]), sqrt_lambda, lambda);
    }
};

// Transforms long enough (Box-Muller: a logarithm, a square root and a sine/cosine per
// pair) that a thread gains from running two units side by side: MTGP32's fill takes two
// units per step of its main loop for these.
template<class F>
struct long_transform : std::false_type
{
};
template<>
struct long_transform<FnNormalF> : std::true_type
{
};
template<>
struct long_transform<FnLogNormalF> : std::true_type
{
};
template<>
struct long_transform<FnNormalD> : std::true_type
{
};
template<>
struct long_transform<FnLogNormalD> : std::true_type
{
};

template<class F>
struct has_table
{
    static constexpr bool value = false;
};
template<>
struct has_table<FnPoisson>
{
    static constexpr bool value = true;
};
template<>
struct has_table<Fn64Poisson>
{
    static constexpr bool value = true;
};
template<class N>
struct has_table<FnMrgRemap<N, FnPoisson>>
{
    static constexpr bool value = true;
};

// Stages a Poisson alias table into shared memory (all threads of the block take part)
// and returns a functor reading it there.  smem holds size doubles then size uints.
template<class F>
struct table_of
{
    __host__ __device__ static F& get(F& f) { return f; }
    __host__ __device__ static const F& get(const F& f) { return f; }
};
template<class N>
struct table_of<FnMrgRemap<N, FnPoisson>>
{
    using W = FnMrgRemap<N, FnPoisson>;
    __host__ __device__ static FnPoisson& get(W& f) { return f.inner; }
    __host__ __device__ static const FnPoisson& get(const W& f) { return f.inner; }
};

template<class F>
__device__ __forceinline__ F stage_table(const F& fw, unsigned char* smem)
{
    if constexpr(has_table<F>::value)
    {
        const auto& f = table_of<F>::get(fw);
        using E       = typename std::remove_cv<typename std::remove_pointer<decltype(f.prob)>::type>::type;
        static_assert(sizeof(E) == 8, "8-byte table entries");
        // packed entries (FnPoisson) carry their aliases; Fn64Poisson has a separate array
        constexpr bool packed = std::is_same<E, unsigned long long>::value;
        E*        p = reinterpret_cast<E*>(smem);
        uint32_t* a = reinterpret_cast<uint32_t*>(smem + sizeof(E) * f.size);
        for(uint32_t i = threadIdx.x; i < f.size; i += blockDim.x)
        {
            p[i] = f.prob[i];
            if constexpr(!packed)
                a[i] = f.alias[i];
        }
        __syncthreads();
        F     g  = fw;
        auto& gt = table_of<F>::get(g);
        gt.prob  = p;
        if constexpr(!packed)
            gt.alias = a;
        return g;
    }
    else
    {
        return fw;
    }
}

template<class F>
inline size_t table_smem_bytes(const F& f)
{
    if constexpr(has_table<F>::value)
    {
        const auto& t = table_of<F>::get(f);
        using E       = typename std::remove_cv<typename std::remove_pointer<decltype(t.prob)>::type>::type;
        constexpr bool packed = std::is_same<E, unsigned long long>::value;
        return (size_t)t.size * (sizeof(E) + (packed ? 0 : sizeof(uint32_t)));
    }
    else
        return 0;
}

// Calls `body(functor)` with the functor that serves distribution d.  Used by every
// generator family to instantiate its kernel once per distribution.
template<class Body>
inline rocrand_status with_functor(Dist d, const DistParams& p, Body&& body)
{
    switch(d)
    {
        case Dist::U32: return body(FnUint{});
        case Dist::U8: return body(FnUchar{});
        case Dist::U16: return body(FnUshort{});
        case Dist::F32: return body(FnFloat{});
        case Dist::F64: return body(FnDouble{});
        case Dist::F16: return body(FnHalf{});
        case Dist::NORMAL_F32: return body(FnNormalF{p.mean_f, p.std_f});
        case Dist::LOGNORMAL_F32: return body(FnLogNormalF{p.mean_f, p.std_f});
        case Dist::NORMAL_F64: return body(FnNormalD{p.mean_d, p.std_d});
        case Dist::LOGNORMAL_F64: return body(FnLogNormalD{p.mean_d, p.std_d});
        case Dist::NORMAL_F16:
            return body(FnNormalH{__half2float(__ushort_as_half(p.mean_h)),
                                  __half2float(__ushort_as_half(p.std_h))});
        case Dist::LOGNORMAL_F16:
            return body(FnLogNormalH{__half2float(__ushort_as_half(p.mean_h)),
                                     __half2float(__ushort_as_half(p.std_h))});
        case Dist::POISSON:
            if(p.huge)
                return body(FnPoissonHuge{p.sqrt_lambda, p.lambda});
            return body(FnPoisson{p.thr, p.alias, p.size, p.offset});
        default: return ROCRAND_STATUS_TYPE_ERROR;
    }
}

// Functor selection for the MRG engines (raw output in [1, m1]).
template<class N, class Body>
inline rocrand_status with_functor_mrg(Dist d, const DistParams& p, Body&& body)
{
    const float mh = __half2float(__ushort_as_half(p.mean_h));
    const float sh = __half2float(__ushort_as_half(p.std_h));
    switch(d)
    {
        case Dist::U32: return body(FnMrgRemap<N, FnUint>{FnUint{}});
        case Dist::U8: return body(FnMrgRemap<N, FnUchar>{FnUchar{}});
        case Dist::U16: return body(FnMrgRemap<N, FnUshort>{FnUshort{}});
        case Dist::F32: return body(FnMrgFloat<N>{});
        case Dist::F64: return body(FnMrgDouble<N>{});
        case Dist::F16: return body(FnMrgRemap<N, FnHalf>{FnHalf{}});
        case Dist::NORMAL_F32: return body(FnMrgNormalF<N>{p.mean_f, p.std_f, false});
        case Dist::LOGNORMAL_F32: return body(FnMrgNormalF<N>{p.mean_f, p.std_f, true});
        case Dist::NORMAL_F64: return body(FnMrgNormalD<N>{p.mean_d, p.std_d, false});
        case Dist::LOGNORMAL_F64: return body(FnMrgNormalD<N>{p.mean_d, p.std_d, true});
        case Dist::NORMAL_F16: return body(FnMrgRemap<N, FnNormalH>{FnNormalH{mh, sh}});
        case Dist::LOGNORMAL_F16: return body(FnMrgRemap<N, FnLogNormalH>{FnLogNormalH{mh, sh}});
        case Dist::POISSON:
            if(p.huge)
                return body(FnMrgPoissonHuge<N>{p.sqrt_lambda, p.lambda});
            return body(FnMrgRemap<N, FnPoisson>{FnPoisson{p.thr, p.alias, p.size, p.offset}});
        default: return ROCRAND_STATUS_TYPE_ERROR;
    }
}

// Functor selection for engines producing 64-bit words.
template<class Body>
inline rocrand_status with_functor64(Dist d, const DistParams& p, Body&& body)
{
    const float mh = __half2float(__ushort_as_half(p.mean_h));
    const float sh = __half2float(__ushort_as_half(p.std_h));
    switch(d)
    {
        case Dist::U64: return body(Fn64Ulonglong{});
        case Dist::U32: return body(Fn64Split<uint32_t, 2>{});
        case Dist::U8: return body(Fn64Split<uint8_t, 8>{});
        case Dist::U16: return body(Fn64Split<uint16_t, 4>{});
        case Dist::F32: return body(Fn64Float{});
        case Dist::F64: return body(Fn64Double{});
        case Dist::F16: return body(Fn64Half{});
        case Dist::NORMAL_F32: return body(Fn64NormalF{p.mean_f, p.std_f, false});
        case Dist::LOGNORMAL_F32: return body(Fn64NormalF{p.mean_f, p.std_f, true});
        case Dist::NORMAL_F64: return body(Fn64NormalD{p.mean_d, p.std_d, false});
        case Dist::LOGNORMAL_F64: return body(Fn64NormalD{p.mean_d, p.std_d, true});
        case Dist::NORMAL_F16: return body(Fn64NormalH{mh, sh, false});
        case Dist::LOGNORMAL_F16: return body(Fn64NormalH{mh, sh, true});
        case Dist::POISSON:
            if(p.huge)
                return body(Fn64PoissonHuge{p.sqrt_lambda, p.lambda});
            return body(Fn64Poisson{p.prob, p.alias, p.size, p.offset});
        default: return ROCRAND_STATUS_TYPE_ERROR;
    }
}

} // namespace rb200
