/*
 * orc_api.c -- generator object and C entry points of the CPU oracle (test
 * infrastructure only).
 *
 * Mirrors library/src/rocrand.cpp:111-449 (NULL handle -> NOT_CREATED, lambda <= 0 ->
 * OUT_OF_RANGE) and the per-generator templates' setters (generator_type.hpp:235-291:
 * set_offset resets; set_seed_uint4 / set_dimensions default to TYPE_ERROR).
 */
#include "orc_internal.h"

static int is_supported(int t)
{
    switch(t)
    {
        case ORC_RNG_PHILOX:
        case ORC_RNG_THREEFRY2_32:
        case ORC_RNG_THREEFRY2_64:
        case ORC_RNG_THREEFRY4_32:
        case ORC_RNG_THREEFRY4_64:
        case ORC_RNG_XORWOW:
        case ORC_RNG_MRG32K3A:
        case ORC_RNG_MRG31K3P:
        case ORC_RNG_LFSR113:
        case ORC_RNG_MT19937:
        case ORC_RNG_MTGP32:
        case ORC_RNG_SOBOL32:
        case ORC_RNG_SCRAMBLED_SOBOL32:
        case ORC_RNG_SOBOL64:
        case ORC_RNG_SCRAMBLED_SOBOL64: return 1;
        default: return 0;
    }
}

int orc_create(orc_gen** out, int rng_type)
{
    if(!out)
        return ORC_OUT_OF_RANGE;
    if(rng_type == ORC_RNG_PSEUDO_DEFAULT)
        rng_type = ORC_RNG_XORWOW;
    if(rng_type == ORC_RNG_QUASI_DEFAULT)
        rng_type = ORC_RNG_SOBOL32;
    if(!is_supported(rng_type))
        return ORC_TYPE_ERROR;
    orc_gen* g = (orc_gen*)calloc(1, sizeof(orc_gen));
    if(!g)
        return ORC_INTERNAL_ERROR;
    g->rng_type = rng_type;
    g->dims     = 1;
    if(rng_type == ORC_RNG_LFSR113)
    {
        /* default seed {2, 8, 16, 128} (lfsr113.hpp:178-186) */
        g->seed4[0] = 2;
        g->seed4[1] = 8;
        g->seed4[2] = 16;
        g->seed4[3] = 128;
    }
    switch(rng_type)
    {
        case ORC_RNG_SOBOL32:
        case ORC_RNG_SCRAMBLED_SOBOL32:
        case ORC_RNG_SOBOL64:
        case ORC_RNG_SCRAMBLED_SOBOL64: g->order = ORC_ORDER_QUASI_DEFAULT; break;
        default: g->order = ORC_ORDER_DEFAULT; break;
    }
    *out = g;
    return ORC_SUCCESS;
}

int orc_destroy(orc_gen* g)
{
    if(g)
    {
        orc_poisson_free(&g->poisson);
        free(g->stf.engines);
        orc_mt19937_free(g);
        orc_mtgp32_free(g);
        free(g);
    }
    return ORC_SUCCESS;
}

int orc_initialize(orc_gen* g)
{
    if(!g)
        return ORC_NOT_CREATED;
    if(g->initialized)
        return ORC_SUCCESS;
    switch(g->rng_type)
    {
        case ORC_RNG_PHILOX: orc_philox_seed(&g->st.philox, g->seed, 0, g->offset); break;
        case ORC_RNG_THREEFRY2_32: orc_threefry_seed(&g->st.threefry, 2, 32, g->seed, g->offset); break;
        case ORC_RNG_THREEFRY2_64: orc_threefry_seed(&g->st.threefry, 2, 64, g->seed, g->offset); break;
        case ORC_RNG_THREEFRY4_32: orc_threefry_seed(&g->st.threefry, 4, 32, g->seed, g->offset); break;
        case ORC_RNG_THREEFRY4_64: orc_threefry_seed(&g->st.threefry, 4, 64, g->seed, g->offset); break;
        case ORC_RNG_XORWOW:
        case ORC_RNG_MRG32K3A:
        case ORC_RNG_MRG31K3P:
        case ORC_RNG_LFSR113:
        {
            const int st = orc_stateful_init(g);
            if(st != ORC_SUCCESS)
                return st;
            break;
        }
        case ORC_RNG_MT19937:
        {
            const int st = orc_mt19937_init(g);
            if(st != ORC_SUCCESS)
                return st;
            break;
        }
        case ORC_RNG_MTGP32:
        {
            const int st = orc_mtgp32_init(g);
            if(st != ORC_SUCCESS)
                return st;
            break;
        }
        case ORC_RNG_SOBOL32:
        case ORC_RNG_SCRAMBLED_SOBOL32:
        case ORC_RNG_SOBOL64:
        case ORC_RNG_SCRAMBLED_SOBOL64: g->sobol_offset = (uint32_t)g->offset; break;
        default: return ORC_TYPE_ERROR;
    }
    g->initialized = 1;
    return ORC_SUCCESS;
}

int orc_set_seed(orc_gen* g, unsigned long long seed)
{
    if(!g)
        return ORC_NOT_CREATED;
    if(g->rng_type == ORC_RNG_LFSR113)
    {
        /* lfsr113.hpp:240-255: overlapping 16-bit shifts, minimums on x and y only */
        g->seed4[0] = (uint32_t)seed;
        g->seed4[1] = (uint32_t)(seed >> 16);
        g->seed4[2] = (uint32_t)(seed >> 32);
        g->seed4[3] = (uint32_t)(seed >> 48);
        if(g->seed4[0] < 2)
            g->seed4[0] += 2;
        if(g->seed4[1] < 8)
            g->seed4[1] += 8;
    }
    else if(g->rng_type == ORC_RNG_MRG32K3A || g->rng_type == ORC_RNG_MRG31K3P)
        seed = seed == 0 ? 12345ull : seed; /* mrg.hpp:236-240 */
    else if(g->rng_type == ORC_RNG_SOBOL32 || g->rng_type == ORC_RNG_SCRAMBLED_SOBOL32
            || g->rng_type == ORC_RNG_SOBOL64 || g->rng_type == ORC_RNG_SCRAMBLED_SOBOL64)
        return ORC_SUCCESS; /* quasi-random generators ignore the seed (sobol.hpp:551-554) */
    g->seed        = seed;
    g->initialized = 0;
    return ORC_SUCCESS;
}

int orc_set_seed_uint4(orc_gen* g, uint32_t x, uint32_t y, uint32_t z, uint32_t w)
{
    if(!g)
        return ORC_NOT_CREATED;
    if(g->rng_type != ORC_RNG_LFSR113)
        return ORC_TYPE_ERROR;
    /* lfsr113.hpp:257-269 */
    g->seed4[0]    = x < 2 ? x + 2 : x;
    g->seed4[1]    = y < 8 ? y + 8 : y;
    g->seed4[2]    = z < 16 ? z + 16 : z;
    g->seed4[3]    = w < 128 ? w + 128 : w;
    g->initialized = 0;
    return ORC_SUCCESS;
}

int orc_set_offset(orc_gen* g, unsigned long long offset)
{
    if(!g)
        return ORC_NOT_CREATED;
    if(g->rng_type == ORC_RNG_MT19937 || g->rng_type == ORC_RNG_MTGP32)
        return ORC_TYPE_ERROR; /* mt19937.hpp:758-763, mtgp32.hpp:389-393 */
    g->offset      = offset;
    g->initialized = 0;
    return ORC_SUCCESS;
}

/* Orderings accepted by a host generator (philox4x32_10.hpp:258-278 and siblings):
 * DYNAMIC is refused on the host. */
int orc_set_ordering(orc_gen* g, int order)
{
    if(!g)
        return ORC_NOT_CREATED;
    if(order == ORC_ORDER_DYNAMIC)
        return ORC_OUT_OF_RANGE;
    int ok = 0;
    switch(g->rng_type)
    {
        case ORC_RNG_XORWOW:
            ok = order == ORC_ORDER_DEFAULT || order == ORC_ORDER_BEST || order == ORC_ORDER_LEGACY
                 || order == ORC_ORDER_SEEDED;
            break;
        case ORC_RNG_SOBOL32:
        case ORC_RNG_SCRAMBLED_SOBOL32:
        case ORC_RNG_SOBOL64:
        case ORC_RNG_SCRAMBLED_SOBOL64: ok = order == ORC_ORDER_QUASI_DEFAULT; break;
        default:
            ok = order == ORC_ORDER_DEFAULT || order == ORC_ORDER_BEST || order == ORC_ORDER_LEGACY;
            break;
    }
    if(!ok)
        return ORC_OUT_OF_RANGE;
    g->order       = order;
    g->initialized = 0;
    return ORC_SUCCESS;
}

static int is_sobol(int t)
{
    return t == ORC_RNG_SOBOL32 || t == ORC_RNG_SCRAMBLED_SOBOL32 || t == ORC_RNG_SOBOL64
           || t == ORC_RNG_SCRAMBLED_SOBOL64;
}

/* sobol.hpp:573-583: 1..20000 dimensions */
int orc_set_dimensions(orc_gen* g, unsigned int dims)
{
    if(!g)
        return ORC_NOT_CREATED;
    if(!is_sobol(g->rng_type))
        return ORC_TYPE_ERROR;
    if(dims < 1 || dims > 20000)
        return ORC_OUT_OF_RANGE;
    g->dims        = dims;
    g->initialized = 0;
    return ORC_SUCCESS;
}

/* ---- generate dispatch ---- */

static int is_threefry64(int t) { return t == ORC_RNG_THREEFRY2_64 || t == ORC_RNG_THREEFRY4_64; }
static int is_threefry(int t)
{
    return t == ORC_RNG_THREEFRY2_32 || t == ORC_RNG_THREEFRY4_32 || is_threefry64(t);
}

static int run(orc_gen* g, void* data, size_t n, const orc_dist* din)
{
    orc_dist d = *din;
    if(is_sobol(g->rng_type))
    {
        /* sobol.hpp:618-640 */
        if(d.kind == D_ULL && (g->rng_type == ORC_RNG_SOBOL32 || g->rng_type == ORC_RNG_SCRAMBLED_SOBOL32))
            return ORC_TYPE_ERROR;
        if(n % g->dims != 0)
            return ORC_LENGTH_NOT_MULTIPLE;
        const int st = orc_initialize(g);
        if(st != ORC_SUCCESS)
            return st;
        if(data == NULL)
            return ORC_SUCCESS;
        return orc_sobol_generate(g, data, n, &d);
    }
    /* 64-bit output only from 64-bit engines (philox4x32_10.hpp:359-375, threefry.hpp:316-321) */
    if(d.kind == D_ULL && !is_threefry64(g->rng_type))
        return ORC_TYPE_ERROR;
    if(is_threefry64(g->rng_type))
        orc_dist_to64(&d);
    /* ThreeFry2x32 serves double normals with the one-word functor (threefry.hpp:441-449) */
    if(g->rng_type == ORC_RNG_THREEFRY2_32 && (d.kind == D_NORMAL_D || d.kind == D_LOGNORMAL_D))
    {
        const double m = d.mean_d, s = d.std_d;
        orc_dist_init(&d, d.kind == D_NORMAL_D ? D_NORMAL_D1 : D_LOGNORMAL_D1);
        d.mean_d = m;
        d.std_d  = s;
    }
    if(g->rng_type == ORC_RNG_MRG31K3P)
        orc_dist_to_mrg(&d, 1);
    if(g->rng_type == ORC_RNG_MRG32K3A)
        orc_dist_to_mrg(&d, 2);
    int st = orc_initialize(g);
    if(st != ORC_SUCCESS)
        return st;
    if(data == NULL)
        return ORC_SUCCESS;
    if(g->rng_type == ORC_RNG_PHILOX)
        return orc_philox_generate(g, data, n, &d);
    if(is_threefry(g->rng_type))
        return orc_threefry_generate(g, data, n, &d);
    if(g->rng_type == ORC_RNG_MT19937)
        return orc_mt19937_generate(g, data, n, &d);
    if(g->rng_type == ORC_RNG_MTGP32)
        return orc_mtgp32_generate(g, data, n, &d);
    return orc_stateful_generate(g, data, n, &d);
}

static int run_kind(orc_gen* g, void* data, size_t n, orc_dist_kind k)
{
    if(!g)
        return ORC_NOT_CREATED;
    orc_dist d;
    orc_dist_init(&d, k);
    return run(g, data, n, &d);
}

int orc_generate(orc_gen* g, uint32_t* out, size_t n) { return run_kind(g, out, n, D_UINT); }

int orc_generate_long_long(orc_gen* g, uint64_t* out, size_t n)
{
    return run_kind(g, out, n, D_ULL);
}

int orc_generate_char(orc_gen* g, uint8_t* out, size_t n) { return run_kind(g, out, n, D_UCHAR); }
int orc_generate_short(orc_gen* g, uint16_t* out, size_t n)
{
    return run_kind(g, out, n, D_USHORT);
}
int orc_generate_uniform(orc_gen* g, float* out, size_t n) { return run_kind(g, out, n, D_FLOAT); }
int orc_generate_uniform_double(orc_gen* g, double* out, size_t n)
{
    return run_kind(g, out, n, D_DOUBLE);
}
int orc_generate_uniform_half(orc_gen* g, uint16_t* out, size_t n)
{
    return run_kind(g, out, n, D_HALF);
}

static int run_normal_f(orc_gen* g, float* out, size_t n, float m, float s, orc_dist_kind k)
{
    if(!g)
        return ORC_NOT_CREATED;
    orc_dist d;
    orc_dist_init(&d, k);
    d.mean_f = m;
    d.std_f  = s;
    return run(g, out, n, &d);
}

static int run_normal_d(orc_gen* g, double* out, size_t n, double m, double s, orc_dist_kind k)
{
    if(!g)
        return ORC_NOT_CREATED;
    orc_dist d;
    orc_dist_init(&d, k);
    d.mean_d = m;
    d.std_d  = s;
    return run(g, out, n, &d);
}

static int run_normal_h(orc_gen* g, uint16_t* out, size_t n, uint16_t m, uint16_t s,
                        orc_dist_kind k)
{
    if(!g)
        return ORC_NOT_CREATED;
    orc_dist d;
    orc_dist_init(&d, k);
    d.mean_h = m;
    d.std_h  = s;
    return run(g, out, n, &d);
}

int orc_generate_normal(orc_gen* g, float* out, size_t n, float mean, float stddev)
{
    return run_normal_f(g, out, n, mean, stddev, D_NORMAL_F);
}
int orc_generate_normal_double(orc_gen* g, double* out, size_t n, double mean, double stddev)
{
    return run_normal_d(g, out, n, mean, stddev, D_NORMAL_D);
}
int orc_generate_normal_half(orc_gen* g, uint16_t* out, size_t n, uint16_t mean, uint16_t stddev)
{
    return run_normal_h(g, out, n, mean, stddev, D_NORMAL_H);
}
int orc_generate_log_normal(orc_gen* g, float* out, size_t n, float mean, float stddev)
{
    return run_normal_f(g, out, n, mean, stddev, D_LOGNORMAL_F);
}
int orc_generate_log_normal_double(orc_gen* g, double* out, size_t n, double mean, double stddev)
{
    return run_normal_d(g, out, n, mean, stddev, D_LOGNORMAL_D);
}
int orc_generate_log_normal_half(orc_gen* g, uint16_t* out, size_t n, uint16_t mean,
                                 uint16_t stddev)
{
    return run_normal_h(g, out, n, mean, stddev, D_LOGNORMAL_H);
}

int orc_generate_poisson(orc_gen* g, uint32_t* out, size_t n, double lambda)
{
    if(!g)
        return ORC_NOT_CREATED;
    if(lambda <= 0.0)
        return ORC_OUT_OF_RANGE;
    orc_dist d;
    const int st = orc_poisson_get(&g->poisson, lambda, &d);
    if(st != ORC_SUCCESS)
        return st;
    return run(g, out, n, &d);
}
