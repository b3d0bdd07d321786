/*
 * make_mt19937_jump.c -- build-time generator of the MT19937 jump polynomials.
 *
 * The reference seeds its 8192 MT19937 generators 2^1000 outputs apart: generator e starts
 * from the seed's state advanced by e * 2^1000 steps (library/src/rng/mt19937.hpp:83-206),
 * using jump polynomials it ships precomputed (rocrand_h_mt19937_jump, made by
 * tools/mt19937_precomputed_generator.cpp from a list in tools/mt19937_precomputed_source.zip).
 * This program derives the same polynomials from the recurrence alone:
 *
 *  1. phi(x), the characteristic polynomial of the MT19937 state transition (degree 19937),
 *     by Berlekamp-Massey over 2 * 19937 + 64 bits of one output bit of the recurrence;
 *  2. q(x) = x^(2^1000) mod phi(x) by 1000 squarings;
 *  3. J_i = q^i mod phi for i = 1..255 (jumps of i * 2^1000 steps) and
 *     K_i = q^(256 i) mod phi for i = 1..31 (jumps of 256 i * 2^1000 steps; 8192 generators
 *     need the second radix-256 digit only up to 31).
 *
 * Output: 286 polynomials of 624 little-endian 32-bit words each (J_1..J_255, K_1..K_31);
 * bit b of word w is the coefficient of x^(32 w + b).  Applying polynomial p to a state s
 * (624 words x_0..x_623 continued by the recurrence) gives the state whose word k is the
 * XOR of x_(i+k) over the set coefficients i of p.
 *
 * Usage: make_mt19937_jump <output.bin>
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MEXP 19937
#define NSTATE 624
#define MTM 397
#define NW 312               /* 64-bit words of a polynomial of degree <= 19967 */
#define PW (2 * NW + 2)      /* words of a product before reduction */
#define NSEQ (2 * MEXP + 64) /* Berlekamp-Massey sequence length */
#define NJ 255
#define NK 31

typedef uint64_t poly[NW + 1];

static uint64_t phi_shift[64][NW + 2]; /* phi << s, s = 0..63 */

static int getbit(const uint64_t* a, long i) { return (int)((a[i >> 6] >> (i & 63)) & 1u); }

/* dst ^= src << shift, src holding nsrc words. */
static void xor_shifted(uint64_t* dst, const uint64_t* src, long nsrc, long shift)
{
    const long w = shift >> 6, s = shift & 63;
    if(s == 0)
    {
        for(long k = 0; k < nsrc; k++)
            dst[w + k] ^= src[k];
        return;
    }
    uint64_t carry = 0;
    for(long k = 0; k < nsrc; k++)
    {
        dst[w + k] ^= (src[k] << s) | carry;
        carry = src[k] >> (64 - s);
    }
    dst[w + nsrc] ^= carry;
}

/* One output bit of the MT19937 recurrence: the top bit of x_(624+n). */
static void mt_bit_sequence(uint64_t* seq)
{
    static uint32_t x[NSTATE + NSEQ + 1];
    x[0] = 5489u;
    for(uint32_t i = 1; i < NSTATE; i++)
        x[i] = 1812433253u * (x[i - 1] ^ (x[i - 1] >> 30)) + i;
    for(long k = 0; k < NSEQ; k++)
    {
        const uint32_t y = (x[k] & 0x80000000u) | (x[k + 1] & 0x7fffffffu);
        x[k + NSTATE]    = x[k + MTM] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    memset(seq, 0, sizeof(uint64_t) * (NSEQ / 64 + 4));
    for(long n = 0; n < NSEQ; n++)
        if(x[NSTATE + n] >> 31)
            seq[n >> 6] |= 1ull << (n & 63);
}

/* Berlekamp-Massey over GF(2); writes phi (monic, degree L) and returns L. */
static long berlekamp_massey(const uint64_t* seq, uint64_t* phi)
{
    /* x^m b spans at most 2 NSEQ bits; every buffer is sized for that */
    const long nwords = 2 * (NSEQ / 64) + 8;
    uint64_t*  rev    = calloc(nwords, sizeof(uint64_t)); /* rev bit k = seq bit NSEQ-1-k */
    uint64_t*  c      = calloc(nwords, sizeof(uint64_t));
    uint64_t*  b      = calloc(nwords, sizeof(uint64_t));
    uint64_t*  t      = calloc(nwords, sizeof(uint64_t));
    if(!rev || !c || !b || !t)
        return -1;
    for(long k = 0; k < NSEQ; k++)
        if(getbit(seq, NSEQ - 1 - k))
            rev[k >> 6] |= 1ull << (k & 63);
    c[0] = b[0] = 1;
    long L = 0, m = 1;
    for(long n = 0; n < NSEQ; n++)
    {
        /* d = sum_{i=0..L} c_i s_(n-i) = parity(c & rev[off .. off+L]), off = NSEQ-1-n */
        const long off = NSEQ - 1 - n, ow = off >> 6, os = off & 63;
        uint64_t   acc = 0;
        for(long w = 0; w <= (L >> 6); w++)
        {
            uint64_t r = rev[ow + w] >> os;
            if(os)
                r |= rev[ow + w + 1] << (64 - os);
            acc ^= c[w] & r;
        }
        if(!__builtin_parityll(acc))
        {
            m++;
            continue;
        }
        const long nb = (n >> 6) + 2;
        if(2 * L <= n)
        {
            memcpy(t, c, sizeof(uint64_t) * nwords);
            xor_shifted(c, b, nb, m);
            L = n + 1 - L;
            memcpy(b, t, sizeof(uint64_t) * nwords);
            m = 1;
        }
        else
        {
            xor_shifted(c, b, nb, m);
            m++;
        }
    }
    /* phi(x) = x^L c(1/x): coefficient of x^(L-i) is c_i */
    memset(phi, 0, sizeof(uint64_t) * (NW + 1));
    for(long i = 0; i <= L && L <= 64 * NW; i++)
        if(getbit(c, i))
            phi[(L - i) >> 6] |= 1ull << ((L - i) & 63);
    free(rev);
    free(c);
    free(b);
    free(t);
    return L;
}

/* acc (degree <= 2 MEXP - 2) reduced mod phi into out. */
static void reduce(uint64_t* acc, uint64_t* out)
{
    for(long d = 2 * MEXP - 2; d >= MEXP; d--)
    {
        if(!getbit(acc, d))
            continue;
        const long      sh  = d - MEXP, w = sh >> 6;
        const uint64_t* src = phi_shift[sh & 63];
        for(long k = 0; k < NW + 2; k++)
            acc[w + k] ^= src[k];
    }
    memcpy(out, acc, sizeof(uint64_t) * NW);
    out[NW] = 0;
}

static void sqrmod(const uint64_t* a, uint64_t* out)
{
    uint64_t acc[PW + NW + 2];
    memset(acc, 0, sizeof(acc));
    for(long w = 0; w < NW; w++)
    {
        for(int h = 0; h < 2; h++)
        {
            uint64_t v = (a[w] >> (32 * h)) & 0xffffffffull, r = 0;
            for(int i = 0; i < 32; i++)
                r |= ((v >> i) & 1ull) << (2 * i);
            acc[2 * w + h] = r;
        }
    }
    reduce(acc, out);
}

static void mulmod(const uint64_t* a, const uint64_t* b, uint64_t* out)
{
    static uint64_t bs[64][NW + 2];
    uint64_t        acc[PW + NW + 2];
    memset(bs, 0, sizeof(bs));
    for(int s = 0; s < 64; s++)
        xor_shifted(bs[s], b, NW, s);
    memset(acc, 0, sizeof(acc));
    for(long i = 0; i < MEXP; i++)
    {
        if(!getbit(a, i))
            continue;
        const uint64_t* src = bs[i & 63];
        const long      w   = i >> 6;
        for(long k = 0; k < NW + 2; k++)
            acc[w + k] ^= src[k];
    }
    reduce(acc, out);
}

static void write_poly(FILE* f, const uint64_t* p)
{
    uint32_t words[NSTATE];
    for(int w = 0; w < NSTATE; w++)
        words[w] = (uint32_t)(p[w / 2] >> (32 * (w & 1)));
    fwrite(words, sizeof(uint32_t), NSTATE, f);
}

int main(int argc, char** argv)
{
    if(argc != 2)
    {
        fprintf(stderr, "usage: %s <output.bin>\n", argv[0]);
        return 2;
    }
    static uint64_t seq[NSEQ / 64 + 8];
    static poly     phi, q, j[NJ + 1], k[NK + 1], big;
    mt_bit_sequence(seq);
    const long L = berlekamp_massey(seq, phi);
    if(L != MEXP)
    {
        fprintf(stderr, "unexpected linear complexity %ld\n", L);
        return 1;
    }
    for(int s = 0; s < 64; s++)
    {
        memset(phi_shift[s], 0, sizeof(phi_shift[s]));
        xor_shifted(phi_shift[s], phi, NW, s);
    }
    memset(q, 0, sizeof(q));
    q[0] = 2; /* x */
    for(int i = 0; i < 1000; i++)
    {
        poly t;
        sqrmod(q, t);
        memcpy(q, t, sizeof(poly));
    }
    memcpy(j[1], q, sizeof(poly));
    for(int i = 2; i <= NJ; i++)
        mulmod(j[i - 1], q, j[i]);
    mulmod(j[NJ], q, big); /* x^(256 * 2^1000) */
    memcpy(k[1], big, sizeof(poly));
    for(int i = 2; i <= NK; i++)
        mulmod(k[i - 1], big, k[i]);
    FILE* f = fopen(argv[1], "wb");
    if(!f)
    {
        perror(argv[1]);
        return 1;
    }
    for(int i = 1; i <= NJ; i++)
        write_poly(f, j[i]);
    for(int i = 1; i <= NK; i++)
        write_poly(f, k[i]);
    if(fclose(f) != 0)
    {
        perror(argv[1]);
        return 1;
    }
    return 0;
}
