/*
 * orc_mt19937.c -- the reference's MT19937 generator restated in plain C (test
 * infrastructure only).
 *
 * library/src/rng/mt19937.hpp and mt19937_octo_engine.hpp:
 *  * 8192 generators (256 blocks x 256 threads, eight threads per generator:
 *    config/config_defaults.hpp:76-80, mt19937.hpp:808); generator e starts from the seed's
 *    state advanced by e * 2^1000 steps (jump_ahead_mt19937, mt19937.hpp:83-206).  The
 *    seed's state is the Knuth initialisation of (seed >> 32) ^ seed (mt19937.hpp:107-116).
 *  * Thread t of a generator owns 78 state words ("slots"): slot 0 is word
 *    {0,113,170,283,340,397,510,567}[t], slot 1+7i+j is word
 *    {1,57,114,171,227,284,341,398,454,511,568}[i] + 7t + j (octo_engine gather).
 *  * Input unit u of a call (one distribution call, iw words) sits at round u / full,
 *    slot group (u % full) / stride, thread u % stride, with stride = 65536 and
 *    full = stride * (78 / iw); round 0 is the state left by the previous call when
 *    start_input > 0 and needs a twist otherwise (generate_short/long_mt19937,
 *    mt19937.hpp:306-662; host bookkeeping mt19937.hpp:910-1042).
 *  * One extra unit serves both head and tail of an unaligned or ragged call; the tail is
 *    written from the top of the unit downwards (mt19937.hpp:404-430).  This follows the
 *    device kernel, where every thread owns its extra-unit flag; the reference's host
 *    emulation of generate_short_mt19937 shares one flag across its eight emulated lanes,
 *    so its head/tail values differ there (the golden fixtures avoid that case).
 * Engine states are computed lazily (only generators a call touches), and twists are
 * applied per generator on first use; the outputs are those of the eager reference.
 */
#include "orc_internal.h"

#define MT_N 624
#define MT_M 397
#define MT_MEXP 19937
#define MT_GENS 8192
#define MT_STRIDE (MT_GENS * 8)
#define MT_SLOTS 78
#define MT_SEQ (MT_MEXP + MT_N - 1)
#define MT_POLY_WORDS 624
#define MT_J 255 /* polynomials for i * 2^1000, i = 1..255 */

extern const uint32_t orc_mt19937_jump_begin[];

struct orc_mt {
    uint32_t* state;  /* [MT_GENS][MT_N], natural word order */
    uint32_t* twists; /* twists applied to each generator */
    uint8_t*  ready;
    uint32_t* digit0; /* [256][MT_N]: seed state advanced by e0 * 2^1000 */
    uint8_t*  d0ready;
    uint32_t* x0; /* MT_SEQ words continuing the seed state */
    uint32_t  seed_state[MT_N];
    uint32_t  global_twists; /* twists every generator has had in the reference */
    uint32_t  start_input;
    uint32_t  prev_iw;
};

static const unsigned kSpecial[8] = {0, 113, 170, 283, 340, 397, 510, 567};
static const unsigned kGroup[11]  = {1, 57, 114, 171, 227, 284, 341, 398, 454, 511, 568};

static unsigned slot_word(unsigned lane, unsigned slot)
{
    if(slot == 0)
        return kSpecial[lane];
    const unsigned i = (slot - 1) / 7, j = (slot - 1) % 7;
    return kGroup[i] + 7 * lane + j;
}

static uint32_t mt_next(uint32_t a, uint32_t b, uint32_t m)
{
    const uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
    return m ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

static void mt_twist(uint32_t* mt)
{
    for(unsigned i = 0; i < MT_N; i++)
        mt[i] = mt_next(mt[i], mt[(i + 1) % MT_N], mt[(i + MT_M) % MT_N]);
}

static uint32_t mt_temper(uint32_t y)
{
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* x[0..623] = s, x[k + 624] by the recurrence, MT_SEQ words in total. */
static void mt_sequence(const uint32_t* s, uint32_t* x)
{
    memcpy(x, s, sizeof(uint32_t) * MT_N);
    for(unsigned k = 0; k + MT_N < MT_SEQ; k++)
        x[k + MT_N] = mt_next(x[k], x[k + 1], x[k + MT_M]);
}

/* Jump polynomial p applied to the state whose continuation is x: word k of the result is
 * the XOR of x[i + k] over the set coefficients i of p (Horner's scheme of
 * mt19937.hpp:147-188 expanded). */
__attribute__((optimize("O3"))) static void mt_apply(const uint32_t* p, const uint32_t* x,
                                                     uint32_t* out)
{
    memset(out, 0, sizeof(uint32_t) * MT_N);
    for(unsigned w = 0; w < MT_POLY_WORDS; w++)
    {
        uint32_t bits = p[w];
        while(bits)
        {
            const unsigned  i   = 32 * w + (unsigned)__builtin_ctz(bits);
            const uint32_t* src = x + i;
            bits &= bits - 1;
            for(unsigned k = 0; k < MT_N; k++)
                out[k] ^= src[k];
        }
    }
}

static const uint32_t* jump_poly(int digit, unsigned value)
{
    const unsigned idx = digit == 0 ? value - 1 : MT_J + value - 1;
    return orc_mt19937_jump_begin + (size_t)idx * MT_POLY_WORDS;
}

static void mt_free(struct orc_mt* m)
{
    if(!m)
        return;
    free(m->state);
    free(m->twists);
    free(m->ready);
    free(m->digit0);
    free(m->d0ready);
    free(m->x0);
    free(m);
}

void orc_mt19937_free(orc_gen* g)
{
    mt_free(g->mt);
    g->mt = NULL;
}

int orc_mt19937_init(orc_gen* g)
{
    orc_mt19937_free(g);
    struct orc_mt* m = (struct orc_mt*)calloc(1, sizeof(struct orc_mt));
    if(!m)
        return ORC_ALLOCATION_FAILED;
    m->state   = (uint32_t*)malloc(sizeof(uint32_t) * MT_N * MT_GENS);
    m->twists  = (uint32_t*)calloc(MT_GENS, sizeof(uint32_t));
    m->ready   = (uint8_t*)calloc(MT_GENS, 1);
    m->digit0  = (uint32_t*)malloc(sizeof(uint32_t) * MT_N * 256);
    m->d0ready = (uint8_t*)calloc(256, 1);
    m->x0      = (uint32_t*)malloc(sizeof(uint32_t) * MT_SEQ);
    if(!m->state || !m->twists || !m->ready || !m->digit0 || !m->d0ready || !m->x0)
    {
        mt_free(m);
        return ORC_ALLOCATION_FAILED;
    }
    const uint32_t seedu = (uint32_t)((g->seed >> 32) ^ g->seed);
    m->seed_state[0]     = seedu;
    for(uint32_t i = 1; i < MT_N; i++)
        m->seed_state[i] = 1812433253u * (m->seed_state[i - 1] ^ (m->seed_state[i - 1] >> 30)) + i;
    mt_sequence(m->seed_state, m->x0);
    g->mt = m;
    return ORC_SUCCESS;
}

static const uint32_t* digit0_state(struct orc_mt* m, unsigned e0)
{
    if(e0 == 0)
        return m->seed_state;
    uint32_t* d = m->digit0 + (size_t)e0 * MT_N;
    if(!m->d0ready[e0])
    {
        mt_apply(jump_poly(0, e0), m->x0, d);
        m->d0ready[e0] = 1;
    }
    return d;
}

/* State of generator e with `twists` twists applied. */
static const uint32_t* generator_state(struct orc_mt* m, unsigned e, uint32_t twists)
{
    uint32_t* s = m->state + (size_t)e * MT_N;
    if(!m->ready[e])
    {
        const uint32_t* d  = digit0_state(m, e % 256);
        const unsigned  e1 = e / 256;
        if(e1 == 0)
            memcpy(s, d, sizeof(uint32_t) * MT_N);
        else
        {
            uint32_t* y = (uint32_t*)malloc(sizeof(uint32_t) * MT_SEQ);
            if(!y)
                abort();
            mt_sequence(d, y);
            mt_apply(jump_poly(1, e1), y, s);
            free(y);
        }
        m->ready[e]  = 1;
        m->twists[e] = 0;
    }
    while(m->twists[e] < twists)
    {
        mt_twist(s);
        m->twists[e]++;
    }
    return s;
}

int orc_mt19937_generate(orc_gen* g, void* data, size_t n, const orc_dist* d)
{
    struct orc_mt* m    = g->mt;
    const unsigned iw   = d->iw, ow = d->ow;
    const uint32_t per  = MT_SLOTS / iw;
    const uint32_t full = MT_STRIDE * per;

    const uintptr_t uptr         = (uintptr_t)data;
    const size_t    misalignment = (ow - uptr / d->tsize % ow) % ow;
    const unsigned  head_size    = (unsigned)orc_min_sz(n, misalignment);
    const unsigned  tail_size    = (unsigned)((n - head_size) % ow);
    const size_t    vec_size     = (n - head_size) / ow;
    const unsigned  extra        = (head_size > 0 || tail_size > 0) ? 1 : 0;
    char*           vec_base     = (char*)data + misalignment * d->tsize;

    /* mt19937.hpp:957-971: a change of input width skips to the next unused slot group */
    if(m->prev_iw != iw && m->start_input > 0)
    {
        const uint32_t used = (m->start_input + MT_STRIDE - 1) / MT_STRIDE * m->prev_iw;
        m->start_input      = (used + iw - 1) / iw * MT_STRIDE;
        if(m->start_input >= full)
            m->start_input = 0;
    }
    const uint32_t start = m->start_input;
    const size_t   total = vec_size + extra;
    const uint32_t first = start == 0 ? 1u : 0u; /* round 0 needs a twist */
    unsigned char  out[8 * 8];
    uint32_t       input[4];

    for(size_t q = 0; q < total; q++)
    {
        const size_t    u     = (size_t)start + q;
        const uint32_t  round = (uint32_t)(u / full);
        const uint32_t  w     = (uint32_t)(u % full);
        const uint32_t  grp   = w / MT_STRIDE;
        const uint32_t  tid   = w % MT_STRIDE;
        const uint32_t* s     = generator_state(m, tid / 8, m->global_twists + round + first);
        for(unsigned i = 0; i < iw; i++)
            input[i] = mt_temper(s[slot_word(tid % 8, grp * iw + i)]);
        orc_dist_apply(d, input, out);
        if(q < vec_size)
        {
            memcpy(vec_base + q * ow * d->tsize, out, (size_t)ow * d->tsize);
            continue;
        }
        for(unsigned o = 0; o < ow; o++)
        {
            if(o < head_size)
                orc_store(d, data, o, out, o);
            if((int)o > (int)ow - (int)tail_size - 1)
                orc_store(d, data, n + (ow - tail_size - 1) - o, out, o);
        }
    }
    if(total > 0)
        m->global_twists += (uint32_t)((start + total - 1) / full) + first;
    m->start_input = (uint32_t)((start + total) % full);
    m->prev_iw     = iw;
    return ORC_SUCCESS;
}
