// precise_math.cuh -- natural logarithm and sine/cosine in double precision whose results
// are correctly rounded except in rare near-halfway cases (internal precision ~2^-66).
//
// The reference's host generators evaluate Box-Muller and the inverse-erf normal with the
// C library's log/sin/cos, which are themselves within ~0.52 ulp of the exact value.  The
// normal and log-normal outputs of this library are compared with them at <= 2 ulp (fp64);
// the device's own 1-2 ulp functions can leave a 3-ulp gap after the products, so the fp64
// transforms use these instead.  Method (standard table-driven reduction, written here):
//  * log x: x = 2^k z with z in [OFF, 2 OFF), OFF just above sqrt(1/2), split by integer
//    operations on the bit pattern; the top 8 bits of z's offset pick one of 256
//    subintervals with a tabulated invc = 1/c of at most 9 significant bits, so that
//    r = z invc - 1 is exact in one fma (|r| < 2^-8; the subinterval around 1 has c = 1);
//    log x = (k ln2_hi + log c_hi) + r - r^2/2 + r^3 P(r) + small terms, the first sums
//    compensated and one final rounding;
//  * sin/cos x (0 <= x <~ 8): x = k pi/2 + r (pi/2 in three parts), |r| = j/64 + b,
//    sin/cos(j/64) from a double-double table, sin b and cos b - 1 by short series.
// Both are IEEE operations only (add, mul, fma, sqrt-free), so host and device builds of
// this header give identical results; the tables are computed in binary128 at build time
// (rocrand_b200/data/make_precise_tables.c).
#pragma once

#include "precise_tables.inc"

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define RB_PM_HD __host__ __device__ __forceinline__
#else
#define RB_PM_HD inline
#endif

namespace rb200
{
namespace pm
{

#if defined(__CUDACC__)
static __device__ const double kLogTabDev[RB_LOG_ROWS * 3] = RB_LOG_INIT;
static __device__ const double kScTabDev[RB_SC_TABLE_ROWS * 4]    = RB_SC_TABLE_INIT;
#endif
static const double kLogTabHost[RB_LOG_ROWS * 3] = RB_LOG_INIT;
static const double kScTabHost[RB_SC_TABLE_ROWS * 4]    = RB_SC_TABLE_INIT;

RB_PM_HD const double* log_table()
{
#if defined(__CUDA_ARCH__)
    return kLogTabDev;
#else
    return kLogTabHost;
#endif
}

RB_PM_HD const double* sc_table()
{
#if defined(__CUDA_ARCH__)
    return kScTabDev;
#else
    return kScTabHost;
#endif
}

// read-only table entry (through the non-coherent cache on the device)
RB_PM_HD double tab(const double* p)
{
#if defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}

RB_PM_HD double fma_(double a, double b, double c)
{
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

RB_PM_HD uint64_t bits_of(double x)
{
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
}

RB_PM_HD double from_bits(uint64_t u)
{
    double x;
    memcpy(&x, &u, 8);
    return x;
}

// s + e == a + b exactly
RB_PM_HD void two_sum(double a, double b, double& s, double& e)
{
    s              = a + b;
    const double bb = s - a;
    e              = (a - (s - bb)) + (b - bb);
}

// s + e == a + b exactly when a == 0 or |a| >= |b| (Dekker's fast two-sum)
RB_PM_HD void fast_two_sum(double a, double b, double& s, double& e)
{
    s = a + b;
    e = b - (s - a);
}

// Natural logarithm, near-correctly rounded.
RB_PM_HD double log(double x)
{
    // The main path runs for every input (the special cases are selected at the end, so
    // that independent calls can interleave): zero, negative, NaN and infinity still give
    // a table row in range there.
    const double x0  = x;
    const bool   sub = x < 0x1p-1022; // subnormal (or zero / negative: replaced below)
    x                = sub ? x * 0x1p54 : x;
    const uint64_t ix  = bits_of(x);
    const uint64_t tmp = ix - RB_LOG_OFF;
    const unsigned i   = static_cast<unsigned>(tmp >> 44) & 255u;
    const int      k   = static_cast<int>(static_cast<int64_t>(tmp) >> 52) - (sub ? 54 : 0);
    const double   z   = from_bits(ix - (tmp & 0xfff0000000000000ull)); // x / 2^k in [OFF, 2 OFF)
    const double*  row = log_table() + 3 * i;
    const double   invc = tab(row), lch = tab(row + 1), lcl = tab(row + 2);
    const double   kd   = static_cast<double>(k);
    const double   r    = fma_(z, invc, -1.0);       // exact: |r| < 2^-8, invc has <= 9 bits
    const double   t1   = fma_(kd, RB_LN2_HI, lch);  // exact: both multiples of 2^-42, |t1| < 2^10
    double         s1, e1, s2, e2;
    two_sum(t1, r, s1, e1);
    // -r^2 / 2 = q + ql exactly
    const double r2 = r * r;
    const double q  = -0.5 * r2;
    const double ql = -0.5 * fma_(r, r, -r2);
    // |s1| >= |q|: s1 = r when t1 = 0 (the subinterval around 1), else |s1| ~ |log x| >= 2^-10
    fast_two_sum(s1, q, s2, e2);
    // r^3 (1/3 - r/4 + r^2/5 - r^3/6 + r^4/7 - r^5/8): the first term left out, r^9/9, is
    // below 2^-67 of the result
    double p = -1.0 / 8.0;
    p        = fma_(p, r, 1.0 / 7.0);
    p        = fma_(p, r, -1.0 / 6.0);
    p        = fma_(p, r, 1.0 / 5.0);
    p        = fma_(p, r, -1.0 / 4.0);
    p        = fma_(p, r, 1.0 / 3.0);
    const double tail = p * (r2 * r);
    const double low  = ((e1 + e2) + (ql + lcl)) + fma_(kd, RB_LN2_LO, tail);
    const double y    = s2 + low;
    return x0 > 0.0 ? (x0 == INFINITY ? x0 : y) : (x0 == 0.0 ? -INFINITY : NAN);
}

// sin and cos of x for 0 <= x < 8 (the Box-Muller angles 0 .. 2 pi), near-correctly rounded.
RB_PM_HD void sincos(double x, double& s_out, double& c_out)
{
    const double kd = rint(x * RB_2_OVER_PI);
    const int    k  = static_cast<int>(kd);
    // r = x - k pi/2 as rh + rl (k pi/2 in three parts; the first two products are exact)
    const double t  = fma_(-kd, RB_PIO2_1, x);
    const double p2 = kd * RB_PIO2_2;
    double       rh, rl;
    two_sum(t, -p2, rh, rl);
    rl = fma_(-kd, RB_PIO2_3, rl);
    {
        const double h = rh + rl;
        rl             = rl - (h - rh);
        rh             = h;
    }
    const bool neg = rh < 0.0;
    rh             = neg ? -rh : rh;
    rl             = neg ? -rl : rl;
    const int     j   = static_cast<int>(rint(rh * 64.0));
    const double* row = sc_table() + 4 * j;
    const double  sh = tab(row), sl = tab(row + 1), ch = tab(row + 2), cl = tab(row + 3);
    const double  bh = rh - static_cast<double>(j) * (1.0 / 64.0); // exact
    const double  bl = rl;
    const double  b2 = bh * bh;
    // sin b - bh = bl + bh^3 (-1/6 + b^2/120 - b^4/5040);  cos b - 1 = -b^2/2 + b^4 (1/24 -
    // b^2/720); |b| <= 2^-7, the first terms left out (b^9/9!, b^8/8!) are below 2^-71
    double sp = -1.0 / 5040.0;
    sp        = fma_(sp, b2, 1.0 / 120.0);
    sp        = fma_(sp, b2, -1.0 / 6.0);
    const double sinb_rest = fma_(sp * b2, bh, bl); // bl + bh^3 S(b^2)
    double       cp        = -1.0 / 720.0;
    cp                     = fma_(cp, b2, 1.0 / 24.0);
    // cos b - 1 = -b^2/2 + b^4 C(b^2), with b^2 including the low part of b
    const double bb  = fma_(2.0 * bh, bl, b2);
    const double cm1 = fma_(cp * bb, bb, -0.5 * bb);
    // sin(a + b) = sin a + (cos a * b + sin a * (cos b - 1) + cos a * (sin b - b))
    const double psh = ch * bh;
    const double psl = fma_(ch, bh, -psh);
    double       ssh, ssl;
    fast_two_sum(sh, psh, ssh, ssl); // sin a >= sin(1/64) > |cos a * b| unless a = 0
    const double s_low = ((ssl + psl) + sl) + fma_(cl, bh, fma_(sh, cm1, ch * sinb_rest));
    const double sv    = ssh + s_low;
    // cos(a + b) = cos a - (sin a * b) + cos a * (cos b - 1) - sin a * (sin b - b)
    const double pch = sh * bh;
    const double pcl = fma_(sh, bh, -pch);
    double       csh, csl;
    fast_two_sum(ch, -pch, csh, csl); // cos a >= 0.7 > |sin a * b|
    const double c_low = ((csl - pcl) + cl) + fma_(-sl, bh, fma_(ch, cm1, -(sh * sinb_rest)));
    const double cv    = csh + c_low;
    const double s     = neg ? -sv : sv;
    // quadrant k: (sin, cos) = (s, c), (c, -s), (-s, -c), (-c, s)
    const bool   odd   = (k & 1) != 0;
    const double so    = odd ? cv : s;
    const double co    = odd ? s : cv;
    s_out              = (k & 2) ? -so : so;
    c_out              = ((k + 1) & 2) ? -co : co;
}

// Natural logarithm of a float, correctly rounded except in rare double-rounding cases.
RB_PM_HD float logf(float x)
{
    return static_cast<float>(log(static_cast<double>(x)));
}

} // namespace pm
} // namespace rb200
