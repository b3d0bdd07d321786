/*
 * orc_dist.c -- distributions of the CPU oracle (test infrastructure only).
 *
 * Restates the reference's host-side distribution functors
 * (library/src/rng/distribution/{uniform,normal,log_normal,poisson,discrete}.hpp) and
 * the scalar conversions they call in the host branch of
 * library/include/rocrand/rocrand_{uniform,normal,discrete}.h.  Built with
 * -ffp-contract=off so every float/double operation rounds as written, as the x86-64
 * host build of the reference does.
 */
#include "orc_internal.h"

#include <math.h>

/* ---- float <-> half, round to nearest even (the host __float2half of cuda_fp16) ---- */
uint16_t orc_float_to_half(float f)
{
    uint32_t x;
    memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t ax   = x & 0x7fffffffu;
    if(ax >= 0x7f800000u)
        return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0u));
    if(ax >= 0x47800000u) /* >= 65536: beyond the largest finite half after rounding */
        return (uint16_t)(sign | 0x7c00u);
    if(ax < 0x38800000u)
    { /* below 2^-14: half subnormal, value = round(|f| * 2^24) ulps of 2^-24 */
        float a;
        memcpy(&a, &ax, 4);
        const float q = rintf(a * 16777216.0f);
        return (uint16_t)(sign | (uint32_t)q);
    }
    const uint32_t e   = (ax >> 23) - 127u + 15u;
    const uint32_t m   = ax & 0x7fffffu;
    uint32_t       h   = (e << 10) | (m >> 13);
    const uint32_t rem = m & 0x1fffu;
    if(rem > 0x1000u || (rem == 0x1000u && (h & 1u)))
        h++;
    return (uint16_t)(sign | h);
}

float orc_half_to_float(uint16_t h)
{
    const uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    const uint32_t e    = (h >> 10) & 0x1fu;
    const uint32_t m    = h & 0x3ffu;
    uint32_t       x;
    if(e == 0)
    {
        const float v = (float)m * 5.9604644775390625e-08f; /* 2^-24 */
        memcpy(&x, &v, 4);
        x |= sign;
    }
    else if(e == 31)
        x = sign | 0x7f800000u | (m << 13);
    else
        x = sign | ((e - 15u + 127u) << 23) | (m << 13);
    float f;
    memcpy(&f, &x, 4);
    return f;
}

/* ---- scalar conversions (rocrand_uniform.h / rocrand_normal.h host branches) ---- */

/* rocrand_uniform.h:61-64 */
static inline float uniform_f(uint32_t v) { return ORC_2POW32_INV + (v * ORC_2POW32_INV); }

/* rocrand_uniform.h:97-107 (two_uints_to_ulong: low word v1, high word v2 >> 11) */
static inline double uniform_d2(uint32_t v1, uint32_t v2)
{
    const uint64_t v = (uint64_t)v1 | ((uint64_t)(v2 >> 11) << 32);
    return ORC_2POW53_INV_DOUBLE + (v * ORC_2POW53_INV_DOUBLE);
}

/* rocrand_uniform.h:92-95 */
static inline double uniform_d1(uint32_t v)
{
    return ORC_2POW32_INV_DOUBLE + (v * ORC_2POW32_INV_DOUBLE);
}

/* rocrand_uniform.h:150-153 */
static inline uint16_t uniform_h(uint16_t v)
{
    return orc_float_to_half(ORC_2POW16_INV + (v * ORC_2POW16_INV));
}

/* rocrand_normal.h:51-66, host branch (sinf/cosf) */
static void box_muller_f(uint32_t x, uint32_t y, float r[2])
{
    const float u = ORC_2POW32_INV + (x * ORC_2POW32_INV);
    const float v = ORC_2POW32_INV_2PI + (y * ORC_2POW32_INV_2PI);
    const float s = sqrtf(-2.0f * logf(u));
    r[0]          = sinf(v) * s;
    r[1]          = cosf(v) * s;
}

/* rocrand_normal.h:68-89, host branch (sin/cos of w*pi) */
static void box_muller_d(uint32_t x, uint32_t y, uint32_t z, uint32_t w, double r[2])
{
    const uint64_t v1 = (uint64_t)x ^ ((uint64_t)y << (53 - 32));
    const double   u  = ORC_2POW53_INV_DOUBLE + (v1 * ORC_2POW53_INV_DOUBLE);
    const uint64_t v2 = (uint64_t)z ^ ((uint64_t)w << (53 - 32));
    const double   ww = (ORC_2POW53_INV_DOUBLE * 2.0) + (v2 * (ORC_2POW53_INV_DOUBLE * 2.0));
    const double   s  = sqrt(-2.0 * orc_log_shift_d(log(u)));
    r[0]              = orc_shift_d(sin(ww * ORC_PI_DOUBLE), orc_trig_ulps) * s;
    r[1]              = orc_shift_d(cos(ww * ORC_PI_DOUBLE), orc_trig_ulps) * s;
}

/* rocrand_normal.h:102-122, branch without half math (the host build) */
static void box_muller_h(uint16_t x, uint16_t y, uint16_t r[2])
{
    const float u = ORC_2POW16_INV + (x * ORC_2POW16_INV);
    const float v = ORC_2POW16_INV_2PI + (y * ORC_2POW16_INV_2PI);
    const float s = sqrtf(-2.0f * logf(u));
    r[0]          = orc_float_to_half(sinf(v) * s);
    r[1]          = orc_float_to_half(cosf(v) * s);
}

int orc_log_ulps  = 0;
int orc_trig_ulps = 0;

void orc_set_libm_ulps(int log_ulps, int trig_ulps)
{
    orc_log_ulps  = log_ulps;
    orc_trig_ulps = trig_ulps;
}

/* rocrand_normal.h:196-220 roc_d_erfinv */
static double erfinv_d(double x)
{
    double tt1, tt2, lnx, sgn;
    sgn = (x < 0.0) ? -1.0 : 1.0;
    x   = (1.0 - x) * (1.0 + x);
    lnx = orc_log_shift_d(log(x));
    if(isnan(lnx))
        return 1.0;
    else if(isinf(lnx))
        return 0.0;
    tt1 = 2.0 / (ORC_PI_DOUBLE * 0.147) + 0.5 * lnx;
    tt2 = 1.0 / (0.147) * lnx;
    return (sgn * sqrt(-tt1 + sqrt(tt1 * tt1 - tt2)));
}

/* rocrand_normal.h:265-270 normal_distribution_double(unsigned int); ROCRAND_SQRT2 is a
 * float literal, promoted to double. */
static double normal_d1(uint32_t x)
{
    const double p = uniform_d1(x);
    return (double)ORC_SQRT2 * erfinv_d(2.0 * p - 1.0);
}

/* rocrand_discrete.h:33-60 discrete_alias with x = r * 2^-32 */
static uint32_t alias_sample(uint32_t r, const orc_dist* d)
{
    const double   x   = r * ORC_2POW32_INV_DOUBLE;
    const double   nx  = d->size * x;
    const double   fnx = floor(nx);
    const double   y   = nx - fnx;
    const uint32_t i   = (uint32_t)fnx;
    return d->offset + (y < d->prob[i] ? i : d->alias[i]);
}

/* rocrand_uniform.h:161-177: MRG raw output in [1, m1] remapped to [0, 2^32);
 * constants of rocrand_mrg31k3p.h:33-34 and rocrand_mrg32k3a.h:39. */
#define ORC_MRG31K3P_UINT32_NORM (2.000000001396983862)
#define ORC_MRG32K3A_UINT_NORM (1.000000048661607)
static inline uint32_t mrg_remap(int mrg, uint32_t v)
{
    if(mrg == 1)
        return (uint32_t)((v - 1) * ORC_MRG31K3P_UINT32_NORM);
    if(mrg == 2)
        return (uint32_t)((v - 1) * ORC_MRG32K3A_UINT_NORM);
    return v;
}

/* MRG normalisation (rocrand_uniform.h:179-219, constants rocrand_mrg31k3p.h:32,
 * rocrand_mrg32k3a.h:38) and Box-Muller over it (rocrand_normal.h:138-172). */
static inline double mrg_norm(int mrg)
{
    return mrg == 1 ? 4.656612875245796923e-10 : 2.3283065498378288e-10;
}
static inline float mrg_f(int mrg, uint32_t v) { return (float)((double)v * mrg_norm(mrg)); }
static void mrg_box_muller_f(int mrg, uint32_t x, uint32_t y, float r[2])
{
    const float u = mrg_f(mrg, x);
    const float v = mrg_f(mrg, y) * ORC_2PI;
    const float s = sqrtf(-2.0f * logf(u));
    r[0]          = sinf(v) * s;
    r[1]          = cosf(v) * s;
}
static void mrg_box_muller_d(int mrg, uint32_t x, uint32_t y, double r[2])
{
    const double u = mrg_f(mrg, x);
    const double v = mrg_f(mrg, y) * 2.0;
    const double s = sqrt(-2.0 * orc_log_shift_d(log(u)));
    r[0]           = orc_shift_d(sin(v * ORC_PI_DOUBLE), orc_trig_ulps) * s;
    r[1]           = orc_shift_d(cos(v * ORC_PI_DOUBLE), orc_trig_ulps) * s;
}

static void mrg_apply(const orc_dist* d, const uint32_t* in, void* outv)
{
    switch(d->kind)
    {
        case D_FLOAT:
        {
            float* o = (float*)outv;
            o[0]     = mrg_f(d->mrg, in[0]);
            return;
        }
        case D_DOUBLE:
        {
            double* o = (double*)outv;
            o[0]      = (double)in[0] * mrg_norm(d->mrg);
            return;
        }
        case D_NORMAL_F:
        case D_LOGNORMAL_F:
        {
            float  r[2];
            float* o = (float*)outv;
            mrg_box_muller_f(d->mrg, in[0], in[1], r);
            for(int k = 0; k < 2; k++)
            {
                const float z = d->mean_f + r[k] * d->std_f;
                o[k]          = d->kind == D_NORMAL_F ? z : expf(z);
            }
            return;
        }
        case D_NORMAL_D:
        case D_LOGNORMAL_D:
        {
            double  r[2];
            double* o = (double*)outv;
            mrg_box_muller_d(d->mrg, in[0], in[1], r);
            for(int k = 0; k < 2; k++)
            {
                const double z = d->mean_d + r[k] * d->std_d;
                o[k]           = d->kind == D_NORMAL_D ? z : exp(z);
            }
            return;
        }
        default: break;
    }
}

/* Distribution shapes on an MRG engine: double uniform takes 1 input, double normals 2. */
void orc_dist_to_mrg(orc_dist* d, int mrg)
{
    d->mrg = mrg;
    if(d->kind == D_DOUBLE)
        d->iw = 1;
    if(d->kind == D_NORMAL_D || d->kind == D_LOGNORMAL_D)
        d->iw = 2;
}

void orc_dist_init(orc_dist* d, orc_dist_kind kind)
{
    memset(d, 0, sizeof(*d));
    d->kind = kind;
    switch(kind)
    {
        case D_UINT: d->iw = 1; d->ow = 1; d->tsize = 4; break;
        case D_UCHAR: d->iw = 1; d->ow = 4; d->tsize = 1; break;
        case D_USHORT: d->iw = 1; d->ow = 2; d->tsize = 2; break;
        case D_FLOAT: d->iw = 1; d->ow = 1; d->tsize = 4; break;
        case D_DOUBLE: d->iw = 2; d->ow = 1; d->tsize = 8; break;
        case D_HALF: d->iw = 1; d->ow = 2; d->tsize = 2; break;
        case D_NORMAL_F:
        case D_LOGNORMAL_F: d->iw = 2; d->ow = 2; d->tsize = 4; break;
        case D_NORMAL_D:
        case D_LOGNORMAL_D: d->iw = 4; d->ow = 2; d->tsize = 8; break;
        case D_NORMAL_H:
        case D_LOGNORMAL_H: d->iw = 1; d->ow = 2; d->tsize = 2; break;
        case D_POISSON:
        case D_POISSON_HUGE: d->iw = 1; d->ow = 1; d->tsize = 4; break;
        case D_NORMAL_D1:
        case D_LOGNORMAL_D1: d->iw = 1; d->ow = 1; d->tsize = 8; break;
        case D_ULL: d->iw = 1; d->ow = 1; d->tsize = 8; break;
    }
}

void orc_dist_apply(const orc_dist* d, const uint32_t* in_raw, void* outv)
{
    /* MRG engines: the single-input distributions see the raw output remapped to
     * [0, 2^32) (uniform.hpp:224-314 via mrg_uniform_distribution_uint); the float/double
     * uniforms and normals have their own formulas. */
    uint32_t        remapped[1];
    const uint32_t* in = in_raw;
    if(d->mrg)
    {
        switch(d->kind)
        {
            case D_FLOAT:
            case D_DOUBLE:
            case D_NORMAL_F:
            case D_NORMAL_D:
            case D_LOGNORMAL_F:
            case D_LOGNORMAL_D: mrg_apply(d, in_raw, outv); return;
            case D_POISSON:
            case D_POISSON_HUGE: break; /* remapped below, in the Poisson cases */
            default:
                remapped[0] = mrg_remap(d->mrg, in_raw[0]);
                in          = remapped;
                break;
        }
    }
    switch(d->kind)
    {
        case D_UINT:
        {
            uint32_t* o = (uint32_t*)outv;
            o[0]        = in[0];
            break;
        }
        case D_UCHAR:
        case D_USHORT: memcpy(outv, &in[0], 4); break;
        case D_FLOAT:
        {
            float* o = (float*)outv;
            o[0]     = uniform_f(in[0]);
            break;
        }
        case D_DOUBLE:
        {
            double* o = (double*)outv;
            o[0]      = uniform_d2(in[0], in[1]);
            break;
        }
        case D_HALF:
        {
            uint16_t* o = (uint16_t*)outv;
            o[0]        = uniform_h((uint16_t)in[0]);
            o[1]        = uniform_h((uint16_t)(in[0] >> 16));
            break;
        }
        case D_NORMAL_F:
        {
            float  r[2];
            float* o = (float*)outv;
            box_muller_f(in[0], in[1], r);
            o[0] = d->mean_f + r[0] * d->std_f;
            o[1] = d->mean_f + r[1] * d->std_f;
            break;
        }
        case D_LOGNORMAL_F:
        {
            float  r[2];
            float* o = (float*)outv;
            box_muller_f(in[0], in[1], r);
            o[0] = expf(d->mean_f + r[0] * d->std_f);
            o[1] = expf(d->mean_f + r[1] * d->std_f);
            break;
        }
        case D_NORMAL_D:
        {
            double  r[2];
            double* o = (double*)outv;
            box_muller_d(in[0], in[1], in[2], in[3], r);
            o[0] = d->mean_d + r[0] * d->std_d;
            o[1] = d->mean_d + r[1] * d->std_d;
            break;
        }
        case D_LOGNORMAL_D:
        {
            double  r[2];
            double* o = (double*)outv;
            box_muller_d(in[0], in[1], in[2], in[3], r);
            o[0] = exp(d->mean_d + r[0] * d->std_d);
            o[1] = exp(d->mean_d + r[1] * d->std_d);
            break;
        }
        case D_NORMAL_H:
        case D_LOGNORMAL_H:
        {
            uint16_t  r[2];
            uint16_t* o = (uint16_t*)outv;
            box_muller_h((uint16_t)in[0], (uint16_t)(in[0] >> 16), r);
            const float m = orc_half_to_float(d->mean_h);
            const float s = orc_half_to_float(d->std_h);
            for(int k = 0; k < 2; k++)
            {
                const float z = m + (s * orc_half_to_float(r[k]));
                o[k]          = orc_float_to_half(d->kind == D_NORMAL_H ? z : expf(z));
            }
            break;
        }
        case D_POISSON:
        {
            uint32_t* o = (uint32_t*)outv;
            o[0]        = alias_sample(mrg_remap(d->mrg, in[0]), d);
            break;
        }
        case D_POISSON_HUGE:
        {
            uint32_t*    o  = (uint32_t*)outv;
            const double nd = normal_d1(mrg_remap(d->mrg, in[0]));
            o[0]            = (uint32_t)round(d->sqrt_lambda * nd + d->lambda);
            break;
        }
        case D_NORMAL_D1:
        {
            double* o = (double*)outv;
            o[0]      = d->mean_d + normal_d1(in[0]) * d->std_d;
            break;
        }
        case D_LOGNORMAL_D1:
        {
            double* o = (double*)outv;
            o[0]      = exp(d->mean_d + normal_d1(in[0]) * d->std_d);
            break;
        }
        case D_ULL: break;
    }
}

void orc_store(const orc_dist* d, void* data, size_t idx, const void* vals, unsigned k)
{
    memcpy((char*)data + idx * d->tsize, (const char*)vals + (size_t)k * d->tsize, d->tsize);
}

/* ---- Poisson tables: poisson.hpp:110-161 (probabilities), discrete.hpp:189-265 ---- */

unsigned orc_poisson_capacity(double lambda)
{
    return (unsigned)(2 * (size_t)(16.0 * (2.0 + sqrt(lambda))));
}

static unsigned poisson_probabilities(double lambda, double* p, unsigned* offset)
{
    const size_t capacity   = 2 * (size_t)(16.0 * (2.0 + sqrt(lambda)));
    const double p_epsilon  = 1e-12;
    const double log_lambda = log(lambda);
    const int    left       = (int)floor(lambda) - (int)(capacity / 2);

    int lo = 0;
    for(int i = (int)(capacity / 2); i >= 0; i--)
    {
        const double x  = left + i;
        const double pp = exp(x * log_lambda - lgamma(x + 1.0) - lambda);
        if(pp < p_epsilon)
        {
            lo = i + 1;
            break;
        }
        p[i] = pp;
    }
    int hi = (int)capacity - 1;
    for(int i = (int)(capacity / 2) + 1; i < (int)capacity; i++)
    {
        const double x  = left + i;
        const double pp = exp(x * log_lambda - lgamma(x + 1.0) - lambda);
        if(pp < p_epsilon)
        {
            hi = i - 1;
            break;
        }
        p[i] = pp;
    }
    for(int i = lo; i <= hi; i++)
        p[i - lo] = p[i];
    *offset = (unsigned)(left + lo);
    return (unsigned)(hi - lo + 1);
}

/* Vose alias construction exactly as discrete.hpp:212-265 (stack order matters). */
static void alias_table(double* p, unsigned size, double* prob, uint32_t* alias)
{
    const double average = 1.0 / size;
    uint32_t*    small   = (uint32_t*)malloc(sizeof(uint32_t) * size);
    uint32_t*    large   = (uint32_t*)malloc(sizeof(uint32_t) * size);
    unsigned     ns = 0, nl = 0;
    for(unsigned i = 0; i < size; i++)
    {
        if(p[i] >= average)
            large[nl++] = i;
        else
            small[ns++] = i;
    }
    while(ns > 0 && nl > 0)
    {
        const uint32_t less = small[--ns];
        const uint32_t more = large[--nl];
        prob[less]          = p[less] * size;
        alias[less]         = more;
        p[more]             = (p[more] + p[less]) - average;
        if(p[more] >= average)
            large[nl++] = more;
        else
            small[ns++] = more;
    }
    for(unsigned i = 0; i < ns; i++)
        prob[small[i]] = 1.0;
    for(unsigned i = 0; i < nl; i++)
        prob[large[i]] = 1.0;
    free(small);
    free(large);
}

unsigned orc_poisson_table(double lambda, double* prob, uint32_t* alias, unsigned* offset)
{
    const unsigned cap = orc_poisson_capacity(lambda);
    double*        p   = (double*)calloc(cap, sizeof(double));
    const unsigned size = poisson_probabilities(lambda, p, offset);
    double         sum  = 0.0;
    for(unsigned i = 0; i < size; i++)
        sum += p[i];
    for(unsigned i = 0; i < size; i++)
        p[i] /= sum;
    alias_table(p, size, prob, alias);
    free(p);
    return size;
}

/* poisson_distribution_manager::get_distribution (poisson.hpp:277-351): tables for
 * lambda <= 4000 (lambda_threshold_huge, rocrand_poisson.h:53), normal approximation above. */
int orc_poisson_get(orc_poisson* pm, double lambda, orc_dist* d)
{
    if(lambda > 4000.0)
    {
        orc_dist_init(d, D_POISSON_HUGE);
        d->lambda      = lambda;
        d->sqrt_lambda = sqrt(lambda);
        return ORC_SUCCESS;
    }
    if(!pm->prob)
    {
        pm->cap   = orc_poisson_capacity(4000.0);
        pm->prob  = (double*)calloc(pm->cap, sizeof(double));
        pm->alias = (uint32_t*)calloc(pm->cap, sizeof(uint32_t));
        pm->cdf   = (double*)calloc(pm->cap, sizeof(double));
        if(!pm->prob || !pm->alias || !pm->cdf)
            return ORC_ALLOCATION_FAILED;
    }
    unsigned offset = 0;
    unsigned size   = 0;
    if(lambda != pm->lambda)
    {
        size = orc_poisson_table(lambda, pm->prob, pm->alias, &offset);
        /* the CDF form (discrete.hpp:275-286) of the same normalised probabilities */
        double* p = (double*)calloc(orc_poisson_capacity(lambda), sizeof(double));
        unsigned off2;
        const unsigned sz2 = poisson_probabilities(lambda, p, &off2);
        double   sum = 0.0;
        for(unsigned i = 0; i < sz2; i++)
            sum += p[i];
        double acc = 0.0;
        for(unsigned i = 0; i < sz2; i++)
        {
            acc += p[i] / sum;
            pm->cdf[i] = acc;
        }
        free(p);
        pm->lambda = lambda;
    }
    else
    {
        double* tmp = (double*)calloc(orc_poisson_capacity(lambda), sizeof(double));
        size        = poisson_probabilities(lambda, tmp, &offset);
        free(tmp);
    }
    orc_dist_init(d, D_POISSON);
    d->prob   = pm->prob;
    d->alias  = pm->alias;
    d->cdf    = pm->cdf;
    d->size   = size;
    d->offset = offset;
    return ORC_SUCCESS;
}

void orc_poisson_free(orc_poisson* pm)
{
    free(pm->prob);
    free(pm->alias);
    free(pm->cdf);
    memset(pm, 0, sizeof(*pm));
}

/* ---- 64-bit engine words (uniform.hpp:119-200, normal.hpp:138-200, log_normal.hpp:138-200,
 *      rocrand_uniform.h:66-69,109-116, rocrand_normal.h:53-58,81-89,124-129,
 *      rocrand_discrete.h:75-81) ---- */

void orc_dist_to64(orc_dist* d)
{
    switch(d->kind)
    {
        case D_ULL: d->iw = 1; d->ow = 1; d->tsize = 8; break;
        case D_UINT: d->iw = 1; d->ow = 2; break;
        case D_UCHAR: d->iw = 1; d->ow = 8; break;
        case D_USHORT: d->iw = 1; d->ow = 4; break;
        case D_FLOAT: d->iw = 1; d->ow = 1; break;
        case D_DOUBLE: d->iw = 1; d->ow = 1; break;
        case D_HALF: d->iw = 1; d->ow = 4; break;
        case D_NORMAL_F:
        case D_LOGNORMAL_F: d->iw = 1; d->ow = 2; break;
        case D_NORMAL_D:
        case D_LOGNORMAL_D: d->iw = 2; d->ow = 2; break;
        case D_NORMAL_H:
        case D_LOGNORMAL_H: d->iw = 1; d->ow = 2; break;
        default: break; /* Poisson: iw1 ow1 */
    }
}

static double uniform_d64(uint64_t v)
{
    return ORC_2POW53_INV_DOUBLE + ((v >> 11) * ORC_2POW53_INV_DOUBLE);
}

void orc_dist_apply64(const orc_dist* d, const uint64_t* in, void* outv)
{
    switch(d->kind)
    {
        case D_ULL:
        case D_UINT:
        case D_UCHAR:
        case D_USHORT: memcpy(outv, &in[0], 8); break;
        case D_FLOAT:
        {
            float* o = (float*)outv;
            o[0]     = ORC_2POW32_INV + ((in[0] >> 32) * ORC_2POW32_INV);
            break;
        }
        case D_DOUBLE:
        {
            double* o = (double*)outv;
            o[0]      = uniform_d64(in[0]);
            break;
        }
        case D_HALF:
        {
            uint16_t* o = (uint16_t*)outv;
            for(int k = 0; k < 4; k++)
                o[k] = uniform_h((uint16_t)(in[0] >> (16 * k)));
            break;
        }
        case D_NORMAL_F:
        case D_LOGNORMAL_F:
        {
            float  r[2];
            float* o = (float*)outv;
            box_muller_f((uint32_t)in[0], (uint32_t)(in[0] >> 32), r);
            for(int k = 0; k < 2; k++)
            {
                const float z = d->mean_f + r[k] * d->std_f;
                o[k]          = d->kind == D_NORMAL_F ? z : expf(z);
            }
            break;
        }
        case D_NORMAL_D:
        case D_LOGNORMAL_D:
        {
            double  r[2];
            double* o = (double*)outv;
            box_muller_d((uint32_t)in[0], (uint32_t)(in[0] >> 32), (uint32_t)in[1],
                         (uint32_t)(in[1] >> 32), r);
            for(int k = 0; k < 2; k++)
            {
                const double z = d->mean_d + r[k] * d->std_d;
                o[k]           = d->kind == D_NORMAL_D ? z : exp(z);
            }
            break;
        }
        case D_NORMAL_H:
        case D_LOGNORMAL_H:
        {
            uint16_t  r[2];
            uint16_t* o = (uint16_t*)outv;
            box_muller_h((uint16_t)in[0], (uint16_t)(in[0] >> 32), r);
            const float m = orc_half_to_float(d->mean_h);
            const float s = orc_half_to_float(d->std_h);
            for(int k = 0; k < 2; k++)
            {
                const float z = m + (s * orc_half_to_float(r[k]));
                o[k]          = orc_float_to_half(d->kind == D_NORMAL_H ? z : expf(z));
            }
            break;
        }
        case D_POISSON:
        {
            /* x = r * 2^-64; r rounds to double first.  When it rounds up to 2^64 the
             * reference indexes one past the table; the index is clamped here. */
            uint32_t*      o   = (uint32_t*)outv;
            const double   x   = in[0] * ORC_2POW64_INV_DOUBLE;
            const double   nx  = d->size * x;
            const double   fnx = floor(nx);
            const double   y   = nx - fnx;
            uint32_t       i   = (uint32_t)fnx;
            if(i >= d->size)
                i = d->size - 1;
            o[0] = d->offset + (y < d->prob[i] ? i : d->alias[i]);
            break;
        }
        case D_POISSON_HUGE:
        {
            uint32_t*    o  = (uint32_t*)outv;
            const double p  = uniform_d64(in[0]);
            const double nd = (double)ORC_SQRT2 * erfinv_d(2.0 * p - 1.0);
            o[0]            = (uint32_t)round(d->sqrt_lambda * nd + d->lambda);
            break;
        }
        default: break;
    }
}
