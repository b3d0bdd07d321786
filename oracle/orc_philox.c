/*
 * orc_philox.c -- Philox4x32-10 host generator restated in C (test infrastructure only).
 *
 * Engine: library/include/rocrand/rocrand_philox4x32_10.h
 *   constants :60-63, seed :134-141, discard_impl :208-218, discard_state :233-243,
 *   bump_counter :252-260, interleave :262-276, ten_rounds :279-291, single_round :295-308.
 * Host kernel body: library/src/rng/philox4x32_10.hpp
 *   next4_leap :88-101, generate_philox :107-214, generator continuity :349-354.
 * The host system runs the body for every (block, thread) of the default NVIDIA config
 * (1024 blocks x 256 threads, config/config_defaults.hpp:54-59), serially
 * (library/src/rng/system.hpp:140-214); this file does the same.
 */
#include "orc_internal.h"

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u
#define PHILOX_BLOCKS 1024u
#define PHILOX_THREADS 256u

static void single_round(uint32_t c[4], const uint32_t k[2])
{
    const uint64_t p0 = (uint64_t)PHILOX_M0 * c[0];
    const uint64_t p1 = (uint64_t)PHILOX_M1 * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t r0 = hi1 ^ c[1] ^ k[0];
    const uint32_t r2 = hi0 ^ c[3] ^ k[1];
    c[0]              = r0;
    c[1]              = lo1;
    c[2]              = r2;
    c[3]              = lo0;
}

static void ten_rounds(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c[4] = {counter[0], counter[1], counter[2], counter[3]};
    uint32_t k[2] = {key[0], key[1]};
    for(int r = 0; r < 9; r++)
    {
        single_round(c, k);
        k[0] += PHILOX_W0;
        k[1] += PHILOX_W1;
    }
    single_round(c, k);
    memcpy(out, c, sizeof(c));
}

static void discard_state_n(orc_philox* e, unsigned long long n)
{
    const uint32_t lo = (uint32_t)n, hi = (uint32_t)(n >> 32);
    uint32_t       t[4];
    memcpy(t, e->counter, sizeof(t));
    e->counter[0] += lo;
    e->counter[1] += hi + (e->counter[0] < t[0] ? 1u : 0u);
    e->counter[2] += (e->counter[1] < t[1] ? 1u : 0u);
    e->counter[3] += (e->counter[2] < t[2] ? 1u : 0u);
}

static void bump_counter(uint32_t c[4])
{
    c[0]++;
    uint32_t add = c[0] == 0 ? 1u : 0u;
    c[1] += add;
    add = c[1] == 0 ? add : 0u;
    c[2] += add;
    add = c[2] == 0 ? add : 0u;
    c[3] += add;
}

static void interleave(uint32_t sub, const uint32_t p[4], const uint32_t q[4], uint32_t out[4])
{
    uint32_t all[8];
    memcpy(all, p, 16);
    memcpy(all + 4, q, 16);
    memcpy(out, all + sub, 16);
}

static void discard_impl(orc_philox* e, unsigned long long offset)
{
    e->substate += (uint32_t)(offset & 3);
    unsigned long long counter_offset = offset / 4;
    counter_offset += e->substate < 4 ? 0 : 1;
    e->substate += e->substate < 4 ? 0 : (uint32_t)-4;
    discard_state_n(e, counter_offset);
}

void orc_philox_discard(orc_philox* e, unsigned long long offset)
{
    discard_impl(e, offset);
    ten_rounds(e->counter, e->key, e->result);
}

void orc_philox_seed(orc_philox* e, unsigned long long seed, unsigned long long subsequence,
                     unsigned long long offset)
{
    e->key[0] = (uint32_t)seed;
    e->key[1] = (uint32_t)(seed >> 32);
    memset(e->counter, 0, sizeof(e->counter));
    memset(e->result, 0, sizeof(e->result));
    e->substate = 0;
    /* discard_subsequence_impl: counter.zw += subsequence */
    {
        const uint32_t lo = (uint32_t)subsequence, hi = (uint32_t)(subsequence >> 32);
        const uint32_t t  = e->counter[2];
        e->counter[2] += lo;
        e->counter[3] += hi + (e->counter[2] < t ? 1u : 0u);
    }
    discard_impl(e, offset);
    ten_rounds(e->counter, e->key, e->result);
}

static uint32_t next(orc_philox* e)
{
    const uint32_t ret = e->result[e->substate];
    e->substate++;
    if(e->substate == 4)
    {
        e->substate = 0;
        bump_counter(e->counter);
        ten_rounds(e->counter, e->key, e->result);
    }
    return ret;
}

static void next4_leap(orc_philox* e, uint32_t leap, uint32_t out[4])
{
    uint32_t ret[4];
    memcpy(ret, e->result, 16);
    if(e->substate > 0)
    {
        uint32_t nc[4], nx[4];
        memcpy(nc, e->counter, 16);
        bump_counter(nc);
        ten_rounds(nc, e->key, nx);
        uint32_t tmp[4];
        interleave(e->substate, ret, nx, tmp);
        memcpy(ret, tmp, 16);
    }
    discard_state_n(e, leap);
    ten_rounds(e->counter, e->key, e->result);
    memcpy(out, ret, 16);
}

/* generate_philox (philox4x32_10.hpp:107-214) for every thread of the default grid. */
int orc_philox_generate(struct orc_gen* g, void* data, size_t n, const orc_dist* d)
{
    const unsigned iw = d->iw, ow = d->ow;
    const unsigned opt               = 4 / iw;
    const unsigned full_output_width = opt * ow;
    const unsigned stride            = PHILOX_BLOCKS * PHILOX_THREADS;

    const uintptr_t uptr         = (uintptr_t)data;
    const size_t    misalignment = (full_output_width - uptr / d->tsize % full_output_width)
                                % full_output_width;
    const unsigned head_size = (unsigned)orc_min_sz(n, misalignment);
    const unsigned tail_size = (unsigned)((n - head_size) % full_output_width);
    const size_t   vec_n     = (n - head_size) / full_output_width;
    char*          vec_base  = (char*)data + misalignment * d->tsize;

    unsigned char out[4][4 * 8];
    uint32_t      input[4];

    for(unsigned tid = 0; tid < stride; tid++)
    {
        /* A thread past vec_n (other than thread 0) writes nothing: skip it. */
        if(tid != 0 && tid > vec_n)
            break;
        orc_philox     e             = g->st.philox;
        const unsigned engine_offset = 4 * tid + (tid == 0 ? 0 : head_size);
        orc_philox_discard(&e, engine_offset);

        if(tid == 0 && head_size > 0)
        {
            for(unsigned s = 0; s < opt; ++s)
            {
                if(s * ow >= head_size)
                    break;
                for(unsigned i = 0; i < iw; ++i)
                    input[i] = next(&e);
                orc_dist_apply(d, input, out[s]);
                for(unsigned o = 0; o < ow; ++o)
                    if(s * ow + o < head_size)
                        orc_store(d, data, s * ow + o, out[s], o);
            }
        }

        size_t index = tid;
        while(index < vec_n)
        {
            uint32_t vs[4];
            next4_leap(&e, stride, vs);
            for(unsigned s = 0; s < opt; s++)
            {
                for(unsigned i = 0; i < iw; i++)
                    input[i] = vs[s * iw + i];
                orc_dist_apply(d, input, out[s]);
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
                orc_dist_apply(d, input, out[s]);
                for(unsigned o = 0; o < ow; ++o)
                    if(s * ow + o < tail_size)
                        orc_store(d, data, n - tail_size + s * ow + o, out[s], o);
            }
        }
    }

    /* Continuity: the host engine advances by the inputs the call consumed. */
    const unsigned long long applied = (unsigned long long)((n + ow - 1) / ow) * iw;
    orc_philox_discard(&g->st.philox, applied);
    return ORC_SUCCESS;
}
