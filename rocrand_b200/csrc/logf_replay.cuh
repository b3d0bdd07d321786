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
// Method.  The kernels evaluate the logarithm L = hi + lo as a pair of floats to about 2^-44
// relative (base(): a table-driven reduction in single precision whose first sums are exact)
// and take f = hi, its rounding to float.  A host result that differs from f can only be f's
// other neighbour on L's side of f (the host's error is below one ulp), and only where L lies
// close to the midpoint between the two.  The build (rocrand_b200/data/make_logf_replay.cpp)
// runs the host's logf over every argument the formula can reach and records
//  * per bucket of arguments (the float's bits >> kBucketShift) and side of f (L below f, L
//    above f), the largest distance of L from the midpoint, in units of 2^-16 ulp (plus one),
//    of an argument whose host result differs from f (0: none);
//  * those arguments, as a set: a bucketed two-choice hash table of 32-bit keys, four per
//    16-byte bucket, so a lookup is two independent 16-byte loads.
// An argument within its bucket's bound for its side tests membership (about 1 % of
// arguments), and a member returns f's neighbour on L's side; all others return f.  The build
// then replays every reachable argument through this same code on the host and requires the
// host's logf result for each.  base() is IEEE float operations only and the distance and
// lookup integer ones, so the host and device builds of this header agree bit for bit.
#pragma once

#include "ieee.cuh"
#include "precise_math.cuh"

#include <cstdint>
#include <cstring>

namespace rb200
{
namespace lr
{

constexpr int      kBucketShift = 15;
constexpr uint32_t kBuckets     = (0x3f800000u >> kBucketShift) + 1; // arguments in (0, 1]
constexpr uint32_t kHash1       = 0x9E3779B1u;                       // Fibonacci hashing
constexpr uint32_t kHash2       = 0x85EBCA77u;

// The tables as the kernels see them (device pointers).
struct Table
{
    const uint32_t* bound        = nullptr; // kBuckets entries: side 0 in bits 0-15, side 1 in 16-31
    const uint4*    keys         = nullptr; // buckets of four member arguments; 0 = empty slot
    uint32_t        log2_buckets = 0;
};

#if defined(__CUDACC__)
static __device__ const float4 kLogfTabDev[RB_LOGF_ROWS] = RB_LOGF_INIT;
#endif
static const float kLogfTabHost[RB_LOGF_ROWS * 4] = RB_LOGF_INIT;

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

// Row i of the float log table: (invc, -log(invc) head, tail, 0).
RB_PM_HD float4 logf_row(uint32_t i)
{
#if defined(__CUDA_ARCH__)
    return __ldg(kLogfTabDev + i);
#else
    return make_float4(kLogfTabHost[4 * i], kLogfTabHost[4 * i + 1], kLogfTabHost[4 * i + 2], 0.0f);
#endif
}

template<class T>
RB_PM_HD T ld(const T* p)
{
#if defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}

// f = the float rounding of log(t) for t in [2^-64, 1], the side of f on which the logarithm
// lies (1: above) and its distance from the midpoint between f and its neighbour on that
// side, in units of 2^-16 ulp of f (0 .. 32768; larger = safer; within one unit).
//   t = 2^k z, z in [OFF, 2 OFF) by integer operations; r = z invc - 1 exact (|r| < 2^-7,
//   invc with at most 8 significant bits); log t = (k ln2_hi + head) + r - r^2/2
//   + r^3 (1/3 - r/4 + r^2/5 - r^3/6) + (tail + k ln2_lo): the first sum exact, the next two
//   compensated (two-sum, exact square), the rest in plain float; r^7/7 is below 2^-44 of
//   the result.
RB_PM_HD float base(float t, uint32_t& dist, uint32_t& side)
{
    const uint32_t ix  = fbits(t);
    const uint32_t tmp = ix - RB_LOGF_OFF;
    const uint32_t i   = (tmp >> 16) & 127u;
    const int      k   = static_cast<int32_t>(tmp) >> 23;
    const float    z   = ffrom(ix - (tmp & 0xff800000u));
    const float4   row = logf_row(i);
    const float    kf  = static_cast<float>(k);
    const float    r   = ieee::ffma(z, row.x, -1.0f);          // exact
    const float    a   = ieee::ffma(kf, RB_LN2F_HI, row.y);    // exact: multiples of 2^-19, |a| < 2^5
    // s1 + e1 = a + r exactly (two-sum)
    const float s1 = ieee::fadd(a, r);
    const float bb = ieee::fsub(s1, a);
    const float e1 = ieee::fadd(ieee::fsub(a, ieee::fsub(s1, bb)), ieee::fsub(r, bb));
    // -r^2 / 2 = q + ql exactly
    const float r2 = ieee::fmul(r, r);
    const float q  = ieee::fmul(-0.5f, r2);
    const float ql = ieee::fmul(-0.5f, ieee::ffma(r, r, -r2));
    // s2 + e2 = s1 + q exactly: |s1| >= |q| (s1 = r when a = 0, else |s1| > 2^-9)
    const float s2 = ieee::fadd(s1, q);
    const float e2 = ieee::fsub(q, ieee::fsub(s2, s1));
    float       p  = ieee::ffma(-1.0f / 6.0f, r, 1.0f / 5.0f);
    p              = ieee::ffma(p, r, -1.0f / 4.0f);
    p              = ieee::ffma(p, r, 1.0f / 3.0f);
    const float tail = ieee::fmul(p, ieee::fmul(r2, r));
    const float low  = ieee::fadd(ieee::fadd(ieee::fadd(e1, e2), ieee::fadd(ql, row.z)),
                                  ieee::ffma(kf, RB_LN2F_LO, tail));
    const float hi = ieee::fadd(s2, low);
    const float lo = ieee::fsub(low, ieee::fsub(hi, s2)); // |lo| <= ulp(hi) / 2
    // |lo| in units of 2^-16 ulp of hi, by a power-of-two scale (exact), and the distance of
    // L from the midpoint half an ulp away.  (Where |hi| is a power of two and lo points
    // inward the midpoint is a quarter of an ulp away; the distance only has to order the
    // arguments, and the build's bounds are taken in this same measure.)
    uint32_t e = (fbits(hi) >> 23) & 0xffu;
    e          = e < 39u ? 39u : e; // hi = 0 (t = 1): lo = 0 too
    const float y = ieee::fmul(fabsf(lo), ffrom((293u - e) << 23)); // |lo| 2^(166 - e)
    dist          = 32768u - static_cast<uint32_t>(y);
    side          = lo > 0.0f ? 1u : 0u;
    return hi;
}

// Key buckets of argument `key` in a table of 2^lb buckets.
RB_PM_HD uint32_t bucket1(uint32_t key, uint32_t lb) { return (key * kHash1) >> (32 - lb); }
RB_PM_HD uint32_t bucket2(uint32_t key, uint32_t lb) { return (key * kHash2) >> (32 - lb); }

// The host C library's logf(t) for an argument of the inverse-erf normal.
RB_PM_HD float logf_host(float t, const Table& tb)
{
    if(!(t >= 0x1p-64f) || !(t <= 1.0f))
        return pm::logf(t); // zero (-inf) and anything outside the formula's range
    uint32_t    dist, side;
    const float    f     = base(t, dist, side);
    const uint32_t key   = fbits(t);
    const uint32_t b2    = ld(tb.bound + (key >> kBucketShift));
    const uint32_t bound = side ? (b2 >> 16) : (b2 & 0xffffu);
    if(dist >= bound)
        return f;
    const uint4 a   = ld(tb.keys + bucket1(key, tb.log2_buckets));
    const uint4 b   = ld(tb.keys + bucket2(key, tb.log2_buckets));
    const bool  hit = (a.x == key) | (a.y == key) | (a.z == key) | (a.w == key) | (b.x == key) | (b.y == key)
                     | (b.z == key) | (b.w == key);
    if(!hit)
        return f;
    // f's neighbour on L's side: one step of the bit pattern, away from zero when L lies
    // beyond f in f's direction
    const uint32_t fb = fbits(f);
    return ffrom((side != 0u) == ((fb >> 31) == 0u) ? fb + 1u : fb - 1u);
}

} // namespace lr
} // namespace rb200
