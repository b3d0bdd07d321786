/*
 * orc_stateful.c -- XORWOW, MRG32k3a, MRG31k3p and LFSR113 host generators restated in C
 * (test infrastructure only).
 *
 * Engines: rocrand_xorwow.h (seed :100-131, next :165-177, discard :134-145),
 * rocrand_mrg32k3a.h (seed :103-120, next :160-190, mod arithmetic :262-300),
 * rocrand_mrg31k3p.h (seed :99-116, next :155-185), rocrand_lfsr113.h (seed :102-110,
 * next :146-160).  Generators: xorwow.hpp:45-161,281-392, mrg.hpp:46-157,284-392,
 * lfsr113.hpp:46-160,240-365 -- E = 131072 engines, engine e = Engine(seed, e,
 * offset/E + (e < start)), output vector j from engine (j + start) % E, the head/tail from
 * the thread with index == vec_n, start += ceil(n/ow) mod E after each call.
 *
 * Skip-ahead: the transition matrices are built here from the engines' recurrences and
 * raised to powers by squaring (GF(2) for XORWOW/LFSR113, 3x3 mod m for the MRGs);
 * engine e is computed as J^e applied to the offset-skipped seeded state, walking e upward
 * one J product at a time (the skips commute, so this equals the reference's
 * subsequence-then-offset order).
 */
#include "orc_internal.h"

#define ST_E 131072u

/* ---------------- engines ---------------- */

static uint32_t next_xorwow(uint32_t* w)
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

static void step_lfsr(uint32_t* z)
{
    uint32_t b;
    b    = ((z[0] << 6) ^ z[0]) >> 13;
    z[0] = ((z[0] & 4294967294u) << 18) ^ b;
    b    = ((z[1] << 2) ^ z[1]) >> 27;
    z[1] = ((z[1] & 4294967288u) << 2) ^ b;
    b    = ((z[2] << 13) ^ z[2]) >> 21;
    z[2] = ((z[2] & 4294967280u) << 7) ^ b;
    b    = ((z[3] << 3) ^ z[3]) >> 12;
    z[3] = ((z[3] & 4294967168u) << 13) ^ b;
}

static uint32_t next_lfsr(uint32_t* z)
{
    step_lfsr(z);
    return z[0] ^ z[1] ^ z[2] ^ z[3];
}

#define M32_M1 4294967087ull
#define M32_M2 4294944443ull

static uint64_t m32_mod_m1(uint64_t p)
{
    p = 209ull * (p >> 32) + (p & 0xffffffffull);
    if(p >= M32_M1)
        p -= M32_M1;
    return p;
}

static uint64_t m32_mod_m2(uint64_t p)
{
    p = 22853ull * (p >> 32) + (p & 0xffffffffull);
    p = 22853ull * (p >> 32) + (p & 0xffffffffull);
    if(p >= M32_M2)
        p -= M32_M2;
    return p;
}

static uint32_t next_mrg32(uint32_t* w)
{
    const uint32_t p1 = (uint32_t)m32_mod_m1(1403580ull * w[1] + 810728ull * (uint32_t)((uint32_t)M32_M1 - w[0]));
    w[0]              = w[1];
    w[1]              = w[2];
    w[2]              = p1;
    const uint32_t p2 = (uint32_t)m32_mod_m2(527612ull * w[5] + 1370589ull * (uint32_t)((uint32_t)M32_M2 - w[3]));
    w[3]              = w[4];
    w[4]              = w[5];
    w[5]              = p2;
    return (p1 - p2) + (p1 <= p2 ? (uint32_t)M32_M1 : 0u);
}

#define M31_M1 2147483647u
#define M31_M2 2147462579u

static uint32_t next_mrg31(uint32_t* w)
{
    uint32_t t = (((w[1] & 511u) << 22) + (w[1] >> 9)) + (((w[2] & 16777215u) << 7) + (w[2] >> 24));
    t -= (t >= M31_M1) ? M31_M1 : 0;
    t += w[2];
    t -= (t >= M31_M1) ? M31_M1 : 0;
    w[2] = w[1];
    w[1] = w[0];
    w[0] = t;
    t    = (((w[3] & 65535u) << 15) + 21069u * (w[3] >> 16));
    t -= (t >= M31_M2) ? M31_M2 : 0;
    t += ((w[5] & 65535u) << 15);
    t -= (t >= M31_M2) ? M31_M2 : 0;
    t += 21069u * (w[5] >> 16);
    t -= (t >= M31_M2) ? M31_M2 : 0;
    t += w[5];
    t -= (t >= M31_M2) ? M31_M2 : 0;
    w[5] = w[4];
    w[4] = w[3];
    w[3] = t;
    return w[0] - w[3] + (w[0] <= w[3] ? M31_M1 : 0);
}

/* ---------------- transition matrices ---------------- */

/* GF(2): n words; row r = image of input bit r. */
typedef struct {
    int      n;
    uint32_t r[160][5];
} gf2m;

static void gf2_apply(const gf2m* m, uint32_t* x)
{
    uint32_t y[5] = {0, 0, 0, 0, 0};
    for(int b = 0; b < m->n * 32; b++)
        if((x[b / 32] >> (b % 32)) & 1u)
            for(int k = 0; k < m->n; k++)
                y[k] ^= m->r[b][k];
    memcpy(x, y, sizeof(uint32_t) * m->n);
}

static void gf2_square(gf2m* m)
{
    gf2m s = *m;
    for(int b = 0; b < m->n * 32; b++)
        gf2_apply(m, s.r[b]);
    *m = s;
}

static void gf2_step_matrix(int kind, gf2m* m)
{
    memset(m, 0, sizeof(*m));
    m->n = kind == ORC_RNG_XORWOW ? 5 : 4;
    for(int b = 0; b < m->n * 32; b++)
    {
        uint32_t x[6] = {0, 0, 0, 0, 0, 0};
        x[b / 32]     = 1u << (b % 32);
        if(kind == ORC_RNG_XORWOW)
        {
            const uint32_t t = x[0] ^ (x[0] >> 2);
            x[0]             = x[1];
            x[1]             = x[2];
            x[2]             = x[3];
            x[3]             = x[4];
            x[4]             = (x[4] ^ (x[4] << 4)) ^ (t ^ (t << 1));
        }
        else
            step_lfsr(x);
        memcpy(m->r[b], x, sizeof(uint32_t) * m->n);
    }
}

/* 3x3 mod m, two components */
typedef struct {
    uint64_t m[2];
    uint64_t a[2][9];
} modm;

static void mod_apply(const modm* t, uint32_t* x)
{
    for(int c = 0; c < 2; c++)
    {
        uint32_t y[3];
        for(int r = 0; r < 3; r++)
        {
            unsigned __int128 s = 0;
            for(int k = 0; k < 3; k++)
                s += (unsigned __int128)t->a[c][r * 3 + k] * x[c * 3 + k];
            y[r] = (uint32_t)(s % t->m[c]);
        }
        memcpy(x + c * 3, y, sizeof(y));
    }
}

static void mod_square(modm* t)
{
    for(int c = 0; c < 2; c++)
    {
        uint64_t s[9];
        for(int r = 0; r < 3; r++)
            for(int k = 0; k < 3; k++)
            {
                unsigned __int128 acc = 0;
                for(int j = 0; j < 3; j++)
                    acc += (unsigned __int128)t->a[c][r * 3 + j] * t->a[c][j * 3 + k];
                s[r * 3 + k] = (uint64_t)(acc % t->m[c]);
            }
        memcpy(t->a[c], s, sizeof(s));
    }
}

static void mod_step_matrix(int kind, modm* t)
{
    memset(t, 0, sizeof(*t));
    if(kind == ORC_RNG_MRG32K3A)
    {
        /* state (x_{n-3}, x_{n-2}, x_{n-1}) */
        t->m[0]    = M32_M1;
        t->a[0][1] = 1;
        t->a[0][5] = 1;
        t->a[0][6] = M32_M1 - 810728;
        t->a[0][7] = 1403580;
        t->m[1]    = M32_M2;
        t->a[1][1] = 1;
        t->a[1][5] = 1;
        t->a[1][6] = M32_M2 - 1370589;
        t->a[1][8] = 527612;
    }
    else
    {
        /* state (x_{n-1}, x_{n-2}, x_{n-3}) */
        t->m[0]    = M31_M1;
        t->a[0][1] = 1u << 22;
        t->a[0][2] = (1u << 7) + 1;
        t->a[0][3] = 1;
        t->a[0][7] = 1;
        t->m[1]    = M31_M2;
        t->a[1][0] = 1u << 15;
        t->a[1][2] = (1u << 15) + 1;
        t->a[1][3] = 1;
        t->a[1][7] = 1;
    }
}

/* Jump data of one family: A^(2^k), k = 0..63 (offsets), and J = A^(2^S) (subsequence). */
typedef struct {
    int   kind;
    gf2m* gp;  /* [64] */
    modm* mp;  /* [64] */
    gf2m  gj;
    modm  mj;
} jumps;

static int      jumps_ready[4];
static jumps    jumps_tab[4];

static int fam_index(int kind)
{
    switch(kind)
    {
        case ORC_RNG_XORWOW: return 0;
        case ORC_RNG_MRG32K3A: return 1;
        case ORC_RNG_MRG31K3P: return 2;
        default: return 3;
    }
}

static const jumps* get_jumps(int kind)
{
    const int i = fam_index(kind);
    if(jumps_ready[i])
        return &jumps_tab[i];
    jumps* j = &jumps_tab[i];
    j->kind  = kind;
    /* subsequence strides: 2^67 (XORWOW), 2^76 (MRG32k3a), 2^72 (MRG31k3p), 2^55 (LFSR113) */
    const int stride_log2 = kind == ORC_RNG_XORWOW ? 67 : kind == ORC_RNG_MRG32K3A ? 76
                                                      : kind == ORC_RNG_MRG31K3P ? 72 : 55;
    if(kind == ORC_RNG_XORWOW || kind == ORC_RNG_LFSR113)
    {
        j->gp = (gf2m*)malloc(sizeof(gf2m) * 64);
        gf2m a;
        gf2_step_matrix(kind, &a);
        for(int k = 0; k < 64; k++)
        {
            j->gp[k] = a;
            gf2_square(&a);
        }
        gf2_step_matrix(kind, &j->gj);
        for(int k = 0; k < stride_log2; k++)
            gf2_square(&j->gj);
    }
    else
    {
        j->mp = (modm*)malloc(sizeof(modm) * 64);
        modm a;
        mod_step_matrix(kind, &a);
        for(int k = 0; k < 64; k++)
        {
            j->mp[k] = a;
            mod_square(&a);
        }
        mod_step_matrix(kind, &j->mj);
        for(int k = 0; k < stride_log2; k++)
            mod_square(&j->mj);
    }
    jumps_ready[i] = 1;
    return j;
}

/* discard(steps) on a state */
static void st_discard(const jumps* j, uint32_t* s, unsigned long long steps)
{
    if(j->kind == ORC_RNG_XORWOW)
        s[5] += (uint32_t)steps * 362437u;
    for(int k = 0; k < 64 && steps; k++, steps >>= 1)
    {
        if(!(steps & 1))
            continue;
        if(j->gp)
            gf2_apply(&j->gp[k], s);
        else
            mod_apply(&j->mp[k], s);
    }
}

static void st_jump_one(const jumps* j, uint32_t* s)
{
    if(j->gp)
        gf2_apply(&j->gj, s);
    else
        mod_apply(&j->mj, s);
}

/* ---------------- seeding ---------------- */

static uint64_t m32_mod_mul(uint32_t i, uint64_t jv, int comp)
{
    long long hi = i / 131072, lo = i - hi * 131072;
    uint64_t (*md)(uint64_t) = comp == 0 ? m32_mod_m1 : m32_mod_m2;
    long long t1 = (long long)(md((uint64_t)hi * jv) * 131072);
    long long t2 = (long long)md((uint64_t)lo * jv);
    lo           = (long long)md((uint64_t)(t1 + t2));
    if(lo < 0)
        lo += (long long)(comp == 0 ? M32_M1 : M32_M2);
    return (uint64_t)lo;
}

static void seeded(const orc_gen* g, uint32_t* s)
{
    unsigned long long seed = g->seed;
    memset(s, 0, sizeof(uint32_t) * 6);
    switch(g->rng_type)
    {
        case ORC_RNG_XORWOW:
        {
            s[0] = 123456789u;
            s[1] = 362436069u;
            s[2] = 521288629u;
            s[3] = 88675123u;
            s[4] = 5783321u;
            s[5] = 6615241u;
            const uint32_t s0 = (uint32_t)seed ^ 0x2c7f967fu;
            const uint32_t s1 = (uint32_t)(seed >> 32) ^ 0xa03697cbu;
            const uint32_t t0 = 1228688033u * s0;
            const uint32_t t1 = 2073658381u * s1;
            s[0] += t0;
            s[1] ^= t0;
            s[2] += t1;
            s[3] ^= t1;
            s[4] += t0;
            s[5] += t1 + t0;
            break;
        }
        case ORC_RNG_MRG32K3A:
        {
            if(seed == 0)
                seed = 12345ull;
            const uint32_t x = (uint32_t)seed ^ 0x55555555u;
            const uint32_t y = (uint32_t)((seed >> 32) ^ 0xAAAAAAAAull);
            s[0]             = (uint32_t)m32_mod_mul(x, seed, 0);
            s[1]             = (uint32_t)m32_mod_mul(y, seed, 0);
            s[2]             = (uint32_t)m32_mod_mul(x, seed, 0);
            s[3]             = (uint32_t)m32_mod_mul(y, seed, 1);
            s[4]             = (uint32_t)m32_mod_mul(x, seed, 1);
            s[5]             = (uint32_t)m32_mod_mul(y, seed, 1);
            break;
        }
        case ORC_RNG_MRG31K3P:
        {
            if(seed == 0)
                seed = 12345ull;
            const uint32_t x = (uint32_t)(seed ^ 0x55555555u);
            const uint32_t y = (uint32_t)((seed >> 32) ^ 0xAAAAAAAAu);
            s[0]             = (uint32_t)((x * seed) % M31_M1);
            s[1]             = (uint32_t)((y * seed) % M31_M1);
            s[2]             = (uint32_t)((x * seed) % M31_M1);
            s[3]             = (uint32_t)((y * seed) % M31_M2);
            s[4]             = (uint32_t)((x * seed) % M31_M2);
            s[5]             = (uint32_t)((y * seed) % M31_M2);
            break;
        }
        default: /* LFSR113: the uint4 seed */
            memcpy(s, g->seed4, sizeof(g->seed4));
            break;
    }
}

int orc_stateful_init(orc_gen* g)
{
    orc_stateful* st = &g->stf;
    if(!st->engines)
    {
        st->engines = (uint32_t*)malloc(sizeof(uint32_t) * 6 * ST_E);
        if(!st->engines)
            return ORC_ALLOCATION_FAILED;
    }
    const jumps*             j     = get_jumps(g->rng_type);
    const unsigned long long jump  = g->offset / ST_E;
    st->start                      = (uint32_t)(g->offset % ST_E);
    uint32_t base0[6], base1[6];
    seeded(g, base0);
    memcpy(base1, base0, sizeof(base0));
    if(g->rng_type == ORC_RNG_LFSR113)
    {
        /* init_lfsr113_engines passes a 32-bit offset (lfsr113.hpp:46-63) */
        st_discard(j, base0, (uint32_t)jump);
        st_discard(j, base1, (uint32_t)((uint32_t)jump + 1u));
    }
    else
    {
        st_discard(j, base0, jump);
        st_discard(j, base1, jump + 1);
    }
    /* engines e >= start from base0, e < start from base1; engine e = J^e base */
    uint32_t cur0[6], cur1[6];
    memcpy(cur0, base0, sizeof(cur0));
    memcpy(cur1, base1, sizeof(cur1));
    for(uint32_t e = 0; e < ST_E; e++)
    {
        memcpy(&st->engines[e * 6], e < st->start ? cur1 : cur0, sizeof(uint32_t) * 6);
        if(e + 1 < ST_E)
        {
            st_jump_one(j, cur0);
            if(e + 1 < st->start)
                st_jump_one(j, cur1);
        }
    }
    return ORC_SUCCESS;
}

static uint32_t engine_next(int kind, uint32_t* w)
{
    switch(kind)
    {
        case ORC_RNG_XORWOW: return next_xorwow(w);
        case ORC_RNG_MRG32K3A: return next_mrg32(w);
        case ORC_RNG_MRG31K3P: return next_mrg31(w);
        default: return next_lfsr(w);
    }
}

/* generate_xorwow / generate_mrg / generate_lfsr113 for every thread of the 512 x 256 grid */
int orc_stateful_generate(orc_gen* g, void* data, size_t n, const orc_dist* d)
{
    orc_stateful*  st = &g->stf;
    const unsigned iw = d->iw, ow = d->ow;
    const uintptr_t uptr         = (uintptr_t)data;
    const size_t    misalignment = (ow - uptr / d->tsize % ow) % ow;
    const unsigned head_size = (unsigned)orc_min_sz(n, misalignment);
    const unsigned tail_size = (unsigned)((n - head_size) % ow);
    const size_t   vec_n     = (n - head_size) / ow;
    char*          vec_base  = (char*)data + misalignment * d->tsize;
    unsigned char  out[8 * 8];
    uint32_t       input[4];

    for(uint32_t tid = 0; tid < ST_E; tid++)
    {
        const int edge = ow > 1 && (vec_n % ST_E) == tid && (head_size > 0 || tail_size > 0);
        if(tid >= vec_n && !edge)
            continue; /* the engine would be loaded and stored back unchanged */
        uint32_t* w     = &st->engines[((tid + st->start) % ST_E) * 6];
        size_t    index = tid;
        while(index < vec_n)
        {
            for(unsigned i = 0; i < iw; i++)
                input[i] = engine_next(g->rng_type, w);
            orc_dist_apply(d, input, out);
            memcpy(vec_base + index * ow * d->tsize, out, (size_t)ow * d->tsize);
            index += ST_E;
        }
        if(ow > 1 && index == vec_n)
        {
            if(head_size > 0)
            {
                for(unsigned i = 0; i < iw; i++)
                    input[i] = engine_next(g->rng_type, w);
                orc_dist_apply(d, input, out);
                for(unsigned o = 0; o < ow; o++)
                    if(o < head_size)
                        orc_store(d, data, o, out, o);
            }
            if(tail_size > 0)
            {
                for(unsigned i = 0; i < iw; i++)
                    input[i] = engine_next(g->rng_type, w);
                orc_dist_apply(d, input, out);
                for(unsigned o = 0; o < ow; o++)
                    if(o < tail_size)
                        orc_store(d, data, n - tail_size + o, out, o);
            }
        }
    }
    st->start = (uint32_t)((st->start + (n + ow - 1) / ow) % ST_E);
    return ORC_SUCCESS;
}
