/*
 * orc_internal.h -- shared definitions of the CPU oracle (test infrastructure only).
 *
 * Status, rng-type and ordering values are the reference's
 * (library/include/rocrand/rocrand.h:59-114).
 */
#ifndef ORC_INTERNAL_H_
#define ORC_INTERNAL_H_

#include "orc.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum {
    ORC_SUCCESS = 0,
    ORC_NOT_CREATED = 101,
    ORC_ALLOCATION_FAILED = 102,
    ORC_TYPE_ERROR = 103,
    ORC_OUT_OF_RANGE = 104,
    ORC_LENGTH_NOT_MULTIPLE = 105,
    ORC_LAUNCH_FAILURE = 107,
    ORC_INTERNAL_ERROR = 108
};

enum {
    ORC_RNG_PSEUDO_DEFAULT = 400,
    ORC_RNG_XORWOW = 401,
    ORC_RNG_MRG32K3A = 402,
    ORC_RNG_MTGP32 = 403,
    ORC_RNG_PHILOX = 404,
    ORC_RNG_MRG31K3P = 405,
    ORC_RNG_LFSR113 = 406,
    ORC_RNG_MT19937 = 407,
    ORC_RNG_THREEFRY2_32 = 408,
    ORC_RNG_THREEFRY2_64 = 409,
    ORC_RNG_THREEFRY4_32 = 410,
    ORC_RNG_THREEFRY4_64 = 411,
    ORC_RNG_QUASI_DEFAULT = 500,
    ORC_RNG_SOBOL32 = 501,
    ORC_RNG_SCRAMBLED_SOBOL32 = 502,
    ORC_RNG_SOBOL64 = 504,
    ORC_RNG_SCRAMBLED_SOBOL64 = 505
};

enum {
    ORC_ORDER_BEST = 100,
    ORC_ORDER_DEFAULT = 101,
    ORC_ORDER_SEEDED = 102,
    ORC_ORDER_LEGACY = 103,
    ORC_ORDER_DYNAMIC = 104,
    ORC_ORDER_QUASI_DEFAULT = 201
};

/* Constants of library/include/rocrand/rocrand_common.h:24-36 (values as the reference
 * spells them; the float ones round to exact powers of two where named so). */
#define ORC_2POW16_INV (1.5258789e-05f)
#define ORC_2POW16_INV_2PI (9.58738e-05f)
#define ORC_2POW32_INV (2.3283064e-10f)
#define ORC_2POW32_INV_DOUBLE (2.3283064365386963e-10)
#define ORC_2POW64_INV (5.4210109e-20f)
#define ORC_2POW64_INV_DOUBLE (5.4210108624275221700372640043497e-20)
#define ORC_2POW32_INV_2PI (1.46291807e-09f)
#define ORC_2POW53_INV_DOUBLE (1.1102230246251565e-16)
#define ORC_PI (3.141592653f)
#define ORC_PI_DOUBLE (3.1415926535897932)
#define ORC_2PI (6.2831855f)
#define ORC_SQRT2 (1.4142135f)
#define ORC_SQRT2_DOUBLE (1.4142135623730951)

/* Distribution kinds (one per reference functor in library/src/rng/distribution/). */
typedef enum {
    D_UINT = 0,     /* uniform_distribution<uint>        iw1 ow1 (uniform.hpp:42-53)  */
    D_UCHAR,        /* uniform_distribution<uchar>       iw1 ow4 (uniform.hpp:55-66)  */
    D_USHORT,       /* uniform_distribution<ushort>      iw1 ow2 (uniform.hpp:68-79)  */
    D_FLOAT,        /* uniform_distribution<float>       iw1 ow1 (uniform.hpp:81-91)  */
    D_DOUBLE,       /* uniform_distribution<double>      iw2 ow1 (uniform.hpp:93-103) */
    D_HALF,         /* uniform_distribution<half>        iw1 ow2 (uniform.hpp:105-117)*/
    D_NORMAL_F,     /* normal_distribution<float,u32,4>  iw2 ow2 (normal.hpp:49-69)   */
    D_NORMAL_D,     /* normal_distribution<double,u32,4> iw4 ow2 (normal.hpp:90-111)  */
    D_NORMAL_H,     /* normal_distribution<half,u32,4>   iw1 ow2 (normal.hpp:113-136) */
    D_LOGNORMAL_F,  /* log_normal_distribution<float>    iw2 ow2 (log_normal.hpp:51-71) */
    D_LOGNORMAL_D,  /* log_normal_distribution<double>   iw4 ow2 (log_normal.hpp:92-113)*/
    D_LOGNORMAL_H,  /* log_normal_distribution<half>     iw1 ow2 (log_normal.hpp:115-139)*/
    D_POISSON,      /* poisson_distribution<ALIAS>       iw1 ow1 (poisson.hpp:49-76)  */
    D_POISSON_HUGE, /* poisson_distribution_huge         iw1 ow1 (poisson.hpp:80-108) */
    D_NORMAL_D1,    /* normal_distribution<double,u32,2> iw1 ow1 (normal.hpp:71-88)   */
    D_LOGNORMAL_D1, /* log_normal_distribution<double,u32,2> iw1 ow1                  */
    D_ULL           /* uniform_distribution<ull,ull>     iw1 ow1 (uniform.hpp:119-130)*/
} orc_dist_kind;

typedef struct orc_dist {
    orc_dist_kind kind;
    unsigned      iw, ow, tsize;
    float         mean_f, std_f;
    double        mean_d, std_d;
    uint16_t      mean_h, std_h;
    /* Poisson */
    const double*   prob;
    const uint32_t* alias;
    const double*   cdf;
    unsigned        size, offset;
    double          lambda, sqrt_lambda;
    /* MRG engines remap raw output before the distribution (see orc_mrg.c) */
    int mrg; /* 0 = none, 1 = mrg31k3p, 2 = mrg32k3a */
} orc_dist;

/* Applies a distribution to iw 32-bit engine outputs, writing ow values of tsize bytes. */
void orc_dist_apply(const orc_dist* d, const uint32_t* in, void* out);
void orc_dist_init(orc_dist* d, orc_dist_kind kind);
/* The same distributions over 64-bit engine words (ThreeFry 2x64/4x64): uniform.hpp:119-200,
 * normal.hpp:138-200, log_normal.hpp:138-200; iw/ow are re-set for 64-bit inputs. */
void orc_dist_to64(orc_dist* d);
void orc_dist_to_mrg(orc_dist* d, int mrg); /* 1 = MRG31k3p, 2 = MRG32k3a */
void orc_dist_apply64(const orc_dist* d, const uint64_t* in, void* out);
void orc_store(const orc_dist* d, void* data, size_t idx, const void* vals, unsigned k);

/* Poisson cache per generator (poisson.hpp:171-412). */
typedef struct {
    double    lambda; /* last lambda whose table is resident, 0 = none */
    double*   prob;
    uint32_t* alias;
    double*   cdf;
    unsigned  cap;
} orc_poisson;

int  orc_poisson_get(orc_poisson* p, double lambda, orc_dist* d);
void orc_poisson_free(orc_poisson* p);

/* Generic "generate one call" entry of a generator family. */
struct orc_gen;
typedef int (*orc_gen_fn)(struct orc_gen* g, void* data, size_t n, const orc_dist* d);

/* Philox engine (rocrand_philox4x32_10.h) */
typedef struct {
    uint32_t counter[4];
    uint32_t result[4];
    uint32_t key[2];
    uint32_t substate;
} orc_philox;

void orc_philox_seed(orc_philox* e, unsigned long long seed, unsigned long long subsequence,
                     unsigned long long offset);
void orc_philox_discard(orc_philox* e, unsigned long long offset);
int  orc_philox_generate(struct orc_gen* g, void* data, size_t n, const orc_dist* d);

/* ThreeFry engines (rocrand_threefry{2,4}_impl.h), words kept in 64-bit storage. */
typedef struct {
    int      dim;  /* 2 or 4 words per block */
    int      bits; /* 32 or 64 */
    uint64_t counter[4];
    uint64_t key[4];
    uint64_t result[4];
    uint32_t substate;
} orc_threefry;

void orc_threefry_seed(orc_threefry* e, int dim, int bits, unsigned long long seed,
                       unsigned long long offset);
int  orc_threefry_generate(struct orc_gen* g, void* data, size_t n, const orc_dist* d);

/* Stateful engines (XORWOW, MRG32k3a, MRG31k3p, LFSR113): 131072 states of 6 words. */
typedef struct {
    uint32_t* engines;
    uint32_t  start;
} orc_stateful;

struct orc_gen;
int orc_stateful_init(struct orc_gen* g);
int orc_stateful_generate(struct orc_gen* g, void* data, size_t n, const orc_dist* d);
int orc_sobol_generate(struct orc_gen* g, void* data, size_t n, const orc_dist* d);

/* MT19937 (orc_mt19937.c): 8192 generators of 624 words, built lazily. */
struct orc_mt;
int  orc_mt19937_init(struct orc_gen* g);
void orc_mt19937_free(struct orc_gen* g);
int  orc_mt19937_generate(struct orc_gen* g, void* data, size_t n, const orc_dist* d);

/* MTGP32 (orc_mtgp32.c): 512 block generators with published parameter sets. */
struct orc_mtgp;
int  orc_mtgp32_init(struct orc_gen* g);
void orc_mtgp32_free(struct orc_gen* g);
int  orc_mtgp32_generate(struct orc_gen* g, void* data, size_t n, const orc_dist* d);

struct orc_gen {
    int                rng_type;
    int                order;
    unsigned long long seed;
    unsigned long long offset;
    int                initialized;
    unsigned           dims;
    orc_poisson        poisson;
    uint32_t           seed4[4]; /* LFSR113 seed */
    uint32_t           sobol_offset; /* 32-bit point counter of the Sobol generators */
    orc_stateful       stf;
    struct orc_mt*     mt;
    struct orc_mtgp*   mtgp;
    union {
        orc_philox   philox;
        orc_threefry threefry;
    } st;
};

static inline size_t orc_min_sz(size_t a, size_t b) { return a < b ? a : b; }

/* Test hook: the host library's logarithm (inside the inverse-erf normal,
 * rocrand_normal.h:174-226, and the fp64 Box-Muller transforms, :68-89, 154-172) and its
 * sine/cosine (fp64 Box-Muller) moved by this many ulps (0 = the reference's values).  A
 * test accepts a device value that equals the reference formula at neighbouring values of
 * these transcendentals: the inverse-erf formula -tt1 + sqrt(tt1^2 - tt2) cancels, and the
 * Box-Muller products can turn one ulp of sin into two of the output. */
extern int orc_log_ulps;
extern int orc_trig_ulps;

static inline float orc_shift_f(float v, int k)
{
    for(; k != 0 && isfinite(v) && v != 0.0f; k += k > 0 ? -1 : 1)
        v = nextafterf(v, k > 0 ? INFINITY : -INFINITY);
    return v;
}

static inline double orc_shift_d(double v, int k)
{
    for(; k != 0 && isfinite(v) && v != 0.0; k += k > 0 ? -1 : 1)
        v = nextafter(v, k > 0 ? INFINITY : -INFINITY);
    return v;
}

static inline float orc_log_shift_f(float v) { return orc_shift_f(v, orc_log_ulps); }
static inline double orc_log_shift_d(double v) { return orc_shift_d(v, orc_log_ulps); }

#endif
