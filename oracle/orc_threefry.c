/*
 * orc_threefry.c -- ThreeFry 2x32/2x64/4x32/4x64-20 host generators restated in C (test
 * infrastructure only).
 *
 * Engines: library/include/rocrand/rocrand_threefry4_impl.h (rotations :62-92, rounds
 * :178-230, discard_impl :232-243, discard_state :256-266, bump_counter :268-278,
 * interleave :280-292), rocrand_threefry2_impl.h (rotations :70-93, rounds :171-208,
 * discard :210-246), seeds rocrand_threefry{2x32,2x64,4x32,4x64}_20.h :85-97.
 * Host kernel body: library/src/rng/threefry.hpp next_leap :66-80, generate_threefry
 * :86-198, continuity :381-386; default grid 1024 x 256 (config_defaults.hpp:68-91).
 * Words of either width are kept in uint64_t and masked for the 32-bit variants.
 */
#include "orc_internal.h"

#define TF_BLOCKS 1024u
#define TF_THREADS 256u

static const int R32x4[8][2] = {{10, 26}, {11, 21}, {13, 27}, {23, 5},
                                {6, 20},  {17, 11}, {25, 10}, {18, 20}};
static const int R64x4[8][2] = {{14, 16}, {52, 57}, {23, 40}, {5, 37},
                                {25, 33}, {46, 12}, {58, 22}, {32, 32}};
static const int R32x2[8]    = {13, 15, 26, 6, 17, 29, 16, 24};
static const int R64x2[8]    = {16, 42, 12, 31, 16, 32, 24, 21};

static uint64_t mask_of(const orc_threefry* e)
{
    return e->bits == 32 ? 0xffffffffull : ~0ull;
}

static uint64_t rotl_w(uint64_t x, int d, int bits, uint64_t m)
{
    return ((x << (d & (bits - 1))) | (x >> ((bits - d) & (bits - 1)))) & m;
}

static void rounds(const orc_threefry* e, const uint64_t* counter, uint64_t* out)
{
    const uint64_t m  = mask_of(e);
    const int      D  = e->dim;
    uint64_t       ks[5];
    uint64_t       X[4];
    ks[D] = e->bits == 32 ? 0x1BD11BDAull : 0x1BD11BDAA9FC1A22ull;
    for(int i = 0; i < D; i++)
    {
        ks[i] = e->key[i];
        ks[D] ^= e->key[i];
        X[i] = (counter[i] + ks[i]) & m;
    }
    for(unsigned r = 0; r < 20; r++)
    {
        if(D == 4)
        {
            const int r0 = e->bits == 32 ? R32x4[r & 7][0] : R64x4[r & 7][0];
            const int r1 = e->bits == 32 ? R32x4[r & 7][1] : R64x4[r & 7][1];
            if((r & 2u) == 0)
            {
                X[0] = (X[0] + X[1]) & m;
                X[1] = rotl_w(X[1], r0, e->bits, m) ^ X[0];
                X[2] = (X[2] + X[3]) & m;
                X[3] = rotl_w(X[3], r1, e->bits, m) ^ X[2];
            }
            else
            {
                X[0] = (X[0] + X[3]) & m;
                X[3] = rotl_w(X[3], r0, e->bits, m) ^ X[0];
                X[2] = (X[2] + X[1]) & m;
                X[1] = rotl_w(X[1], r1, e->bits, m) ^ X[2];
            }
        }
        else
        {
            const int r0 = e->bits == 32 ? R32x2[r & 7] : R64x2[r & 7];
            X[0]         = (X[0] + X[1]) & m;
            X[1]         = rotl_w(X[1], r0, e->bits, m) ^ X[0];
        }
        if((r & 3u) == 3)
        {
            const unsigned inj = r / 4;
            for(int i = 0; i < D; i++)
                X[i] = (X[i] + ks[(i + 1 + inj) % (D + 1)]) & m;
            X[D - 1] = (X[D - 1] + 1 + inj) & m;
        }
    }
    memcpy(out, X, sizeof(uint64_t) * D);
}

/* discard_state(offset): 4x32 adds (lo, hi) words with carries; 64-bit words add the
 * offset to word 0 and carry; 2x32 is a 64-bit counter. */
static void discard_state_n(orc_threefry* e, unsigned long long off)
{
    const uint64_t m = mask_of(e);
    uint64_t       old[4];
    memcpy(old, e->counter, sizeof(old));
    if(e->bits == 32)
    {
        const uint64_t lo = off & 0xffffffffull, hi = off >> 32;
        e->counter[0] = (e->counter[0] + lo) & m;
        e->counter[1] = (e->counter[1] + hi + (e->counter[0] < old[0] ? 1 : 0)) & m;
        if(e->dim == 4)
        {
            e->counter[2] = (e->counter[2] + (e->counter[1] < old[1] ? 1 : 0)) & m;
            e->counter[3] = (e->counter[3] + (e->counter[2] < old[2] ? 1 : 0)) & m;
        }
    }
    else
    {
        e->counter[0] += off;
        e->counter[1] += (e->counter[0] < old[0] ? 1 : 0);
        if(e->dim == 4)
        {
            e->counter[2] += (e->counter[1] < old[1] ? 1 : 0);
            e->counter[3] += (e->counter[2] < old[2] ? 1 : 0);
        }
    }
}

static void bump(const orc_threefry* e, uint64_t* c)
{
    const uint64_t m = mask_of(e);
    c[0]             = (c[0] + 1) & m;
    uint64_t add     = c[0] == 0 ? 1 : 0;
    for(int i = 1; i < e->dim; i++)
    {
        c[i] = (c[i] + add) & m;
        add  = c[i] == 0 ? add : 0;
    }
}

static void discard_impl(orc_threefry* e, unsigned long long off)
{
    const unsigned D = (unsigned)e->dim;
    e->substate += (uint32_t)(off & (D - 1));
    unsigned long long co = off / D;
    co += e->substate < D ? 0 : 1;
    e->substate -= e->substate < D ? 0 : D;
    discard_state_n(e, co);
}

static void discard(orc_threefry* e, unsigned long long off)
{
    discard_impl(e, off);
    rounds(e, e->counter, e->result);
}

void orc_threefry_seed(orc_threefry* e, int dim, int bits, unsigned long long seed,
                       unsigned long long offset)
{
    memset(e, 0, sizeof(*e));
    e->dim  = dim;
    e->bits = bits;
    const uint64_t m = mask_of(e);
    if(dim == 4)
        for(int i = 0; i < 4; i++)
            e->key[i] = (seed >> (16 * i)) & m;
    else
    {
        e->key[0] = seed & m;
        e->key[1] = (seed >> 32) & m;
    }
    discard(e, offset);
    rounds(e, e->counter, e->result);
}

static uint64_t next(orc_threefry* e)
{
    const uint64_t ret = e->result[e->substate];
    e->substate++;
    if(e->substate == (uint32_t)e->dim)
    {
        e->substate = 0;
        bump(e, e->counter);
        rounds(e, e->counter, e->result);
    }
    return ret;
}

static void next_leap(orc_threefry* e, unsigned leap, uint64_t* out)
{
    uint64_t ret[8];
    memcpy(ret, e->result, sizeof(uint64_t) * e->dim);
    if(e->substate > 0)
    {
        uint64_t nc[4], nx[4];
        memcpy(nc, e->counter, sizeof(nc));
        bump(e, nc);
        rounds(e, nc, nx);
        memcpy(ret + e->dim, nx, sizeof(uint64_t) * e->dim);
        memmove(ret, ret + e->substate, sizeof(uint64_t) * e->dim);
    }
    discard_state_n(e, leap);
    rounds(e, e->counter, e->result);
    memcpy(out, ret, sizeof(uint64_t) * e->dim);
}

static void apply(const orc_dist* d, int bits, const uint64_t* in, void* out)
{
    if(bits == 64)
        orc_dist_apply64(d, in, out);
    else
    {
        uint32_t w[4];
        for(unsigned i = 0; i < d->iw; i++)
            w[i] = (uint32_t)in[i];
        orc_dist_apply(d, w, out);
    }
}

/* generate_threefry (threefry.hpp:86-198) for every thread of the default grid. */
int orc_threefry_generate(struct orc_gen* g, void* data, size_t n, const orc_dist* d)
{
    const unsigned D = (unsigned)g->st.threefry.dim;
    const int      bits = g->st.threefry.bits;
    const unsigned iw = d->iw, ow = d->ow;
    const unsigned opt               = D / iw;
    const unsigned full_output_width = opt * ow;
    const unsigned stride            = TF_BLOCKS * TF_THREADS;

    const uintptr_t uptr         = (uintptr_t)data;
    const size_t    misalignment = (full_output_width - uptr / d->tsize % full_output_width)
                                % full_output_width;
    const unsigned head_size = (unsigned)orc_min_sz(n, misalignment);
    const unsigned tail_size = (unsigned)((n - head_size) % full_output_width);
    const size_t   vec_n     = (n - head_size) / full_output_width;
    char*          vec_base  = (char*)data + misalignment * d->tsize;

    unsigned char out[4][8 * 8];
    uint64_t      input[4];

    for(unsigned tid = 0; tid < stride; tid++)
    {
        if(tid != 0 && tid > vec_n)
            break;
        orc_threefry   e             = g->st.threefry;
        const unsigned engine_offset = D * tid + (tid == 0 ? 0 : head_size / ow * iw);
        discard(&e, engine_offset);

        if(tid == 0 && head_size > 0)
        {
            for(unsigned s = 0; s < opt; ++s)
            {
                if(s * ow >= head_size)
                    break;
                for(unsigned i = 0; i < iw; ++i)
                    input[i] = next(&e);
                apply(d, bits, input, out[s]);
                for(unsigned o = 0; o < ow; ++o)
                    if(s * ow + o < head_size)
                        orc_store(d, data, s * ow + o, out[s], o);
            }
        }

        size_t index = tid;
        while(index < vec_n)
        {
            uint64_t vs[4];
            next_leap(&e, stride, vs);
            for(unsigned s = 0; s < opt; s++)
            {
                apply(d, bits, vs + s * iw, out[s]);
                memcpy(vec_base + (index * full_output_width + s * ow) * d->tsize, out[s],
                       (size_t)ow * d->tsize);
            }
            index += stride;
        }

        if(index == vec_n && tail_size > 0)
        {
            for(unsigned s = 0; s < opt; ++s)
            {
                if(s * ow >= tail_size)
                    break;
                for(unsigned i = 0; i < iw; ++i)
                    input[i] = next(&e);
                apply(d, bits, input, out[s]);
                for(unsigned o = 0; o < ow; ++o)
                    if(s * ow + o < tail_size)
                        orc_store(d, data, n - tail_size + s * ow + o, out[s], o);
            }
        }
    }

    const unsigned long long applied = (unsigned long long)((n + ow - 1) / ow) * iw;
    discard(&g->st.threefry, applied);
    return ORC_SUCCESS;
}
