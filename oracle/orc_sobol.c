/*
 * orc_sobol.c -- Sobol32/64, plain and scrambled, host generators restated in C (test
 * infrastructure only).
 *
 * Direction vectors: the Joe-Kuo recurrence (tools/sobol_utils.hpp:76-106) over the
 * per-dimension parameters embedded from rocrand_b200/data/sobol_params.bin; scrambled
 * tables add 640000 (32-bit) / 1280000 (64-bit) to every word
 * (tools/scrambled_sobol{32,64}_direction_vector_generator.cpp).
 * Engine: rocrand_sobol32.h / rocrand_sobol64.h (Gray-code state, discard :134-138), scrambled
 * variants XOR with the constant (rocrand_scrambled_sobol32.h:40-58); the generator takes the
 * scramble constant of dimension d from word d of its own direction table (sobol.hpp:514).
 * Generation (sobol.hpp:155-256, 618-717): out[d * N + i] = dist(value at offset + i), the
 * 32-bit point counter advancing by N per call.  The leap-frog of the reference's threads
 * visits the same points, so this restatement steps each dimension sequentially.
 * Distributions: sobol_*_distribution (uniform.hpp:351-442, normal.hpp:272-330,
 * log_normal.hpp:296-370) and the CDF Poisson (rocrand_discrete.h:92-115).
 */
#include "orc_internal.h"

#define SOBOL_DIMS 20000u

extern const unsigned char orc_sobol_params_begin[];

static uint32_t* g_v32[2]; /* plain, scrambled */
static uint64_t* g_v64[2];

static uint32_t bits_get(const unsigned char* p, size_t* pos, int n)
{
    uint32_t v = 0;
    for(int i = 0; i < n; i++, (*pos)++)
        v |= (uint32_t)((p[*pos / 8] >> (*pos % 8)) & 1u) << i;
    return v;
}

static void build_tables(void)
{
    if(g_v32[0])
        return;
    for(int k = 0; k < 2; k++)
    {
        g_v32[k] = (uint32_t*)calloc((size_t)SOBOL_DIMS * 32, 4);
        g_v64[k] = (uint64_t*)calloc((size_t)SOBOL_DIMS * 64, 8);
    }
    for(int j = 0; j < 32; j++)
        g_v32[0][j] = 1u << (31 - j);
    for(int j = 0; j < 64; j++)
        g_v64[0][j] = 1ull << (63 - j);
    const unsigned char* blob = orc_sobol_params_begin + 12; /* magic + count */
    size_t               pos  = 0;
    for(unsigned d = 1; d < SOBOL_DIMS; d++)
    {
        const uint32_t s = bits_get(blob, &pos, 5);
        const uint32_t a = bits_get(blob, &pos, (int)s - 1);
        uint32_t       m[32];
        for(uint32_t j = 0; j < s; j++)
            m[j] = bits_get(blob, &pos, (int)j + 1);
        uint32_t* v = g_v32[0] + (size_t)d * 32;
        uint64_t* w = g_v64[0] + (size_t)d * 64;
        for(uint32_t j = 0; j < s; j++)
        {
            v[j] = m[j] << (31 - j);
            w[j] = (uint64_t)m[j] << (63 - j);
        }
        for(uint32_t j = s; j < 64; j++)
        {
            uint64_t x = w[j - s] ^ (w[j - s] >> s);
            for(uint32_t k = 1; k < s; k++)
                if((a >> (s - 1 - k)) & 1u)
                    x ^= w[j - k];
            w[j] = x;
            if(j < 32)
            {
                uint32_t y = v[j - s] ^ (v[j - s] >> s);
                for(uint32_t k = 1; k < s; k++)
                    if((a >> (s - 1 - k)) & 1u)
                        y ^= v[j - k];
                v[j] = y;
            }
        }
    }
    for(size_t i = 0; i < (size_t)SOBOL_DIMS * 32; i++)
        g_v32[1][i] = g_v32[0][i] + 640000u;
    for(size_t i = 0; i < (size_t)SOBOL_DIMS * 64; i++)
        g_v64[1][i] = g_v64[0][i] + 1280000ull;
}

static int rzb(uint64_t x, int bits)
{
    /* rightmost zero bit of x (0 for all ones, as the device engine does) */
    for(int b = 0; b < bits; b++)
        if(!((x >> b) & 1u))
            return b;
    return 0;
}

static float erfinv_f(float x)
{
    float tt1, tt2, lnx, sgn;
    sgn = (x < 0.0f) ? -1.0f : 1.0f;
    x   = (1.0f - x) * (1.0f + x);
    lnx = orc_log_shift_f(logf(x));
    if(isnan(lnx))
        return 1.0f;
    else if(isinf(lnx))
        return 0.0f;
    tt1 = 2.0f / (ORC_PI * 0.147f) + 0.5f * lnx;
    tt2 = 1.0f / (0.147f) * lnx;
    return (sgn * sqrtf(-tt1 + sqrtf(tt1 * tt1 - tt2)));
}

static double erfinv_dd(double x)
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

static float normal_f(uint32_t hi32)
{
    const float p = ORC_2POW32_INV + (hi32 * ORC_2POW32_INV);
    return ORC_SQRT2 * erfinv_f(2.0f * p - 1.0f);
}

static double u_d(uint64_t x, int is64)
{
    if(is64)
        return ORC_2POW53_INV_DOUBLE + ((x >> 11) * ORC_2POW53_INV_DOUBLE);
    return ORC_2POW32_INV_DOUBLE + ((uint32_t)x * ORC_2POW32_INV_DOUBLE);
}

static double normal_d(uint64_t x, int is64)
{
    const double p = u_d(x, is64);
    return (double)ORC_SQRT2 * erfinv_dd(2.0 * p - 1.0);
}

static uint32_t cdf_sample(double x, const orc_dist* d)
{
    unsigned min = 0, max = d->size - 1;
    do
    {
        const unsigned center = (min + max) / 2;
        if(x > d->cdf[center])
            min = center + 1;
        else
            max = center;
    }
    while(min != max);
    return d->offset + min;
}

static void sobol_value(const orc_dist* d, uint64_t x, int is64, void* out)
{
    const int      B  = is64 ? 64 : 32;
    const uint32_t hi = (uint32_t)(x >> (B - 32));
    switch(d->kind)
    {
        case D_UINT: *(uint32_t*)out = hi; break;
        case D_ULL: *(uint64_t*)out = x; break;
        case D_UCHAR: *(uint8_t*)out = (uint8_t)(x >> (B - 8)); break;
        case D_USHORT: *(uint16_t*)out = (uint16_t)(x >> (B - 16)); break;
        case D_FLOAT: *(float*)out = ORC_2POW32_INV + (hi * ORC_2POW32_INV); break;
        case D_DOUBLE: *(double*)out = u_d(x, is64); break;
        case D_HALF:
        {
            const uint16_t s = (uint16_t)(x >> (B - 16));
            *(uint16_t*)out  = orc_float_to_half(ORC_2POW16_INV + (s * ORC_2POW16_INV));
            break;
        }
        case D_NORMAL_F: *(float*)out = d->mean_f + normal_f(hi) * d->std_f; break;
        case D_LOGNORMAL_F: *(float*)out = expf(d->mean_f + (d->std_f * normal_f(hi))); break;
        case D_NORMAL_D: *(double*)out = d->mean_d + normal_d(x, is64) * d->std_d; break;
        case D_LOGNORMAL_D: *(double*)out = exp(d->mean_d + (d->std_d * normal_d(x, is64))); break;
        case D_NORMAL_H:
        {
            const float v   = normal_f(hi);
            *(uint16_t*)out = orc_float_to_half(orc_half_to_float(d->mean_h) + v * orc_half_to_float(d->std_h));
            break;
        }
        case D_LOGNORMAL_H:
        {
            const float v   = normal_f(hi);
            *(uint16_t*)out = orc_float_to_half(expf(orc_half_to_float(d->mean_h) + (orc_half_to_float(d->std_h) * v)));
            break;
        }
        case D_POISSON:
        {
            const double xd = is64 ? (double)x * ORC_2POW64_INV_DOUBLE : (uint32_t)x * ORC_2POW32_INV_DOUBLE;
            *(uint32_t*)out = cdf_sample(xd, d);
            break;
        }
        case D_POISSON_HUGE:
        {
            const double nd = normal_d(x, is64);
            *(uint32_t*)out = (uint32_t)round(d->sqrt_lambda * nd + d->lambda);
            break;
        }
        default: break;
    }
}

int orc_sobol_generate(orc_gen* g, void* data, size_t n, const orc_dist* d)
{
    build_tables();
    const int is64      = g->rng_type == ORC_RNG_SOBOL64 || g->rng_type == ORC_RNG_SCRAMBLED_SOBOL64;
    const int scrambled = g->rng_type == ORC_RNG_SCRAMBLED_SOBOL32 || g->rng_type == ORC_RNG_SCRAMBLED_SOBOL64;
    const size_t N      = n / g->dims;
    for(unsigned dim = 0; dim < g->dims; dim++)
    {
        char* row = (char*)data + (size_t)dim * N * d->tsize;
        if(is64)
        {
            const uint64_t* v  = g_v64[scrambled] + (size_t)dim * 64;
            const uint64_t  c  = scrambled ? g_v64[1][dim] : 0;
            uint64_t        i  = (uint64_t)g->sobol_offset;
            const uint64_t  gr = i ^ (i >> 1);
            uint64_t        x  = 0;
            for(int b = 0; b < 64; b++)
                if((gr >> b) & 1u)
                    x ^= v[b];
            for(size_t k = 0; k < N; k++)
            {
                sobol_value(d, x ^ c, 1, row + k * d->tsize);
                x ^= v[rzb(i, 64)];
                i++;
            }
        }
        else
        {
            const uint32_t* v  = g_v32[scrambled] + (size_t)dim * 32;
            const uint32_t  c  = scrambled ? g_v32[1][dim] : 0;
            uint32_t        i  = g->sobol_offset;
            const uint32_t  gr = i ^ (i >> 1);
            uint32_t        x  = 0;
            for(int b = 0; b < 32; b++)
                if((gr >> b) & 1u)
                    x ^= v[b];
            for(size_t k = 0; k < N; k++)
            {
                sobol_value(d, (uint64_t)(x ^ c), 0, row + k * d->tsize);
                x ^= v[rzb(i, 32)];
                i++;
            }
        }
    }
    g->sobol_offset += (uint32_t)N;
    return ORC_SUCCESS;
}
