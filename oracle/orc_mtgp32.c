/*
 * orc_mtgp32.c -- the reference's MTGP32 generator restated in plain C (test infrastructure
 * only).
 *
 * library/src/rng/mtgp32.hpp:232-305 and library/include/rocrand/rocrand_mtgp32.h:
 *  * 512 generators (one per block of 256 threads, config/config_defaults.hpp:48-52), each
 *    with its own published parameter set (rocrand_mtgp32_11213.h, read from
 *    rocrand_b200/data/mtgp32_params.bin) and a 1024-word state ring, seeded by
 *    rocrand_make_state_mtgp32 (seed ^= seed >> 32; generator i gets (uint32)seed + i + 1,
 *    rocrand_mtgp32_init_state);
 *  * one engine step: r = para_rec(s[k], s[k+1], s[k+pos]), s[k+351] = r, output
 *    temper(r, s[k+pos-1]), k advancing by one (the device does 256 steps at once);
 *  * output vector j comes from generator (j / 256) % 512, thread j % 256, call round
 *    j / 131072; each distribution call takes its iw inputs from iw successive block steps;
 *    after the full rounds every generator steps once more if the last round is partial
 *    (writing only what exists), and once more if the call has a head or tail, written by
 *    the threads at vector indices vec_n_up and vec_n_up + 1 (generate_mtgp).
 */
#include "orc_internal.h"

#define MTGP_N 351
#define MTGP_STATE 1024
#define MTGP_MASK 1023
#define MTGP_GENS 512
#define MTGP_BLOCK 256
#define MTGP_WORDS 36 /* pos, sh1, sh2, tbl[16], tmp_tbl[16], mask */

extern const unsigned char orc_mtgp32_params_begin[];

struct orc_mtgp {
    uint32_t status[MTGP_GENS][MTGP_STATE];
    int      offset[MTGP_GENS];
};

static const uint32_t* params_of(int g)
{
    return (const uint32_t*)(orc_mtgp32_params_begin + 12) + (size_t)g * MTGP_WORDS;
}

void orc_mtgp32_free(orc_gen* g)
{
    free(g->mtgp);
    g->mtgp = NULL;
}

int orc_mtgp32_init(orc_gen* g)
{
    orc_mtgp32_free(g);
    struct orc_mtgp* m = (struct orc_mtgp*)calloc(1, sizeof(struct orc_mtgp));
    if(!m)
        return ORC_ALLOCATION_FAILED;
    const unsigned long long seed = g->seed ^ (g->seed >> 32);
    for(int i = 0; i < MTGP_GENS; i++)
    {
        /* rocrand_mtgp32_init_state: 351 words from the seed and the hidden seed */
        const uint32_t* p      = params_of(i);
        const uint32_t* tbl    = p + 3;
        uint32_t        hidden = tbl[4] ^ (tbl[8] << 16);
        uint32_t        tmp    = hidden;
        tmp += tmp >> 16;
        tmp += tmp >> 8;
        const uint32_t fill = (tmp & 0xffu) * 0x01010101u;
        uint32_t*      a    = m->status[i];
        for(int k = 0; k < MTGP_N; k++)
            a[k] = fill;
        a[0] = (uint32_t)seed + (uint32_t)i + 1u;
        a[1] = hidden;
        for(uint32_t k = 1; k < MTGP_N; k++)
            a[k] ^= 1812433253u * (a[k - 1] ^ (a[k - 1] >> 30)) + k;
        m->offset[i] = 0;
    }
    g->mtgp = m;
    return ORC_SUCCESS;
}

static uint32_t mtgp_next(struct orc_mtgp* m, int g)
{
    const uint32_t* p     = params_of(g);
    const uint32_t  pos   = p[0], sh1 = p[1], sh2 = p[2];
    const uint32_t* tbl   = p + 3;
    const uint32_t* tmp   = p + 19;
    const uint32_t  mask  = p[35];
    uint32_t*       s     = m->status[g];
    const int       k     = m->offset[g];
    /* para_rec (rocrand_mtgp32.h) */
    uint32_t x = (s[k & MTGP_MASK] & mask) ^ s[(k + 1) & MTGP_MASK];
    uint32_t y = s[(k + (int)pos) & MTGP_MASK];
    x ^= x << sh1;
    y      = x ^ (y >> sh2);
    const uint32_t r = y ^ tbl[y & 0x0f];
    s[(k + MTGP_N) & MTGP_MASK] = r;
    /* temper */
    uint32_t t = s[(k + (int)pos - 1) & MTGP_MASK];
    t ^= t >> 16;
    t ^= t >> 8;
    m->offset[g] = (k + 1) & MTGP_MASK;
    return r ^ tmp[t & 0x0f];
}

int orc_mtgp32_generate(orc_gen* g, void* data, size_t n, const orc_dist* d)
{
    struct orc_mtgp* m  = g->mtgp;
    const unsigned   iw = d->iw, ow = d->ow;
    const uintptr_t  uptr         = (uintptr_t)data;
    const size_t     misalignment = (ow - uptr / d->tsize % ow) % ow;
    const size_t     head_size    = orc_min_sz(n, misalignment);
    const size_t     tail_size    = (n - head_size) % ow;
    const size_t     vec_n        = (n - head_size) / ow;
    const size_t     rem          = vec_n % MTGP_BLOCK;
    const size_t     vec_n_down   = vec_n - rem;
    const size_t     vec_n_up     = rem == 0 ? vec_n_down : vec_n_down + MTGP_BLOCK;
    const size_t     stride       = (size_t)MTGP_GENS * MTGP_BLOCK;
    char*            vec_base     = (char*)data + misalignment * d->tsize;
    static uint32_t  in[MTGP_BLOCK][4];
    static unsigned char out[MTGP_BLOCK][64];

    for(int b = 0; b < MTGP_GENS; b++)
    {
        size_t index = (size_t)b * MTGP_BLOCK;
        int    phase = 0; /* 0 full rounds, 1 partial round, 2 head/tail, 3 done */
        while(phase < 3)
        {
            if(phase == 0 && index >= vec_n_down)
                phase = 1;
            if(phase == 1 && index >= vec_n_up)
                phase = 2;
            if(phase == 2 && !(ow > 1 && (head_size > 0 || tail_size > 0)))
                break;
            /* one block step per input word, thread order within a step */
            for(unsigned i = 0; i < iw; i++)
                for(int t = 0; t < MTGP_BLOCK; t++)
                    in[t][i] = mtgp_next(m, b);
            for(int t = 0; t < MTGP_BLOCK; t++)
            {
                orc_dist_apply(d, in[t], out[t]);
                const size_t idx = index + (size_t)t;
                if(phase < 2)
                {
                    if(idx < vec_n)
                        memcpy(vec_base + idx * ow * d->tsize, out[t], (size_t)ow * d->tsize);
                    continue;
                }
                /* save_head_tail (mtgp32.hpp) */
                if(idx == vec_n_up)
                    for(unsigned o = 0; o < ow; o++)
                        if(o < head_size)
                            orc_store(d, data, o, out[t], o);
                if(idx == vec_n_up + 1)
                    for(unsigned o = 0; o < ow; o++)
                        if(o < tail_size)
                            orc_store(d, data, n - tail_size + o, out[t], o);
            }
            index += stride;
            if(phase == 1 || phase == 2)
                phase++;
        }
    }
    return ORC_SUCCESS;
}
