/*
 * make_xorwow_jump.c -- build-time generator of the XORWOW subsequence jump polynomials.
 *
 * A fresh XORWOW generator gives engine e the seed's state advanced by e subsequences of
 * 2^67 steps (library/src/rng/xorwow.hpp:45-61 with rocrand_xorwow.h:134-164; the Weyl
 * counter is unchanged by such a jump, 2^67 * 362437 being 0 mod 2^32).  The xorshift part
 * of the step is a linear map A on 160 bits, so
 *
 *     A^(e 2^67) s = p_e(A) s,   p_e(x) = x^(e 2^67) mod phi(x),
 *
 * phi being the characteristic polynomial of A (degree 160).  And A^k s is the state after
 * k steps, the window (s_k, ..., s_(k+4)) of the word sequence that the recurrence continues
 * from s_0..s_4 = s.  So engine e's state word j is the XOR of s_(k+j) over the set
 * coefficients k of p_e: a sum of windows of one 164-word sequence per seed, with p_e
 * independent of the seed.  This program derives the p_e from the recurrence alone:
 *
 *  1. phi by Berlekamp-Massey over 2 * 160 + 64 bits of one bit of the word sequence;
 *  2. q = x^(2^67) mod phi by 67 squarings;
 *  3. p_0 = 1, p_(e+1) = p_e q mod phi for e < 131072 (the engines of one generator);
 *  4. a self-check: for a random state and several e, the window sum of p_e equals the
 *     state moved by (A^(2^67))^e computed with 160 x 160 GF(2) matrices; any mismatch
 *     fails the build.
 *
 * Output: 5 x 131072 little-endian 32-bit words, word-major: word j of p_e (coefficients
 * x^(32 j) .. x^(32 j + 31)) at index j * 131072 + e, so that a warp reading consecutive e
 * makes one coalesced load per word.
 *
 * Usage: make_xorwow_jump <output.bin>
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define DEG 160
#define ENGINES 131072
#define NSEQ (2 * DEG + 64)
#define SEQW (DEG + 4)

typedef struct
{
    uint64_t w[6]; /* up to 384 coefficients */
} poly;

static int getbit(const uint64_t* a, int i) { return (int)((a[i >> 6] >> (i & 63)) & 1u); }

static void xorwow_step(uint32_t* x)
{
    const uint32_t t = x[0] ^ (x[0] >> 2);
    x[0]             = x[1];
    x[1]             = x[2];
    x[2]             = x[3];
    x[3]             = x[4];
    x[4]             = (x[4] ^ (x[4] << 4)) ^ (t ^ (t << 1));
}

/* The word sequence s_0..s_(n-1) continued from a state. */
static void word_sequence(const uint32_t* s0, uint32_t* seq, int n)
{
    uint32_t x[5];
    memcpy(x, s0, sizeof(x));
    for(int k = 0; k < 5 && k < n; k++)
        seq[k] = x[k];
    for(int k = 5; k < n; k++)
    {
        xorwow_step(x);
        seq[k] = x[4];
    }
}

/* Berlekamp-Massey over GF(2) on bits seq[0..NSEQ); returns L and phi (monic, degree L). */
static int berlekamp_massey(const int* s, poly* phi)
{
    int c[NSEQ + 1], b[NSEQ + 1], t[NSEQ + 1];
    memset(c, 0, sizeof(c));
    memset(b, 0, sizeof(b));
    c[0] = b[0] = 1;
    int L = 0, m = 1;
    for(int n = 0; n < NSEQ; n++)
    {
        int d = s[n];
        for(int i = 1; i <= L; i++)
            d ^= c[i] & s[n - i];
        if(!d)
        {
            m++;
            continue;
        }
        if(2 * L <= n)
        {
            memcpy(t, c, sizeof(c));
            for(int i = 0; i + m <= NSEQ; i++)
                c[i + m] ^= b[i];
            L = n + 1 - L;
            memcpy(b, t, sizeof(b));
            m = 1;
        }
        else
        {
            for(int i = 0; i + m <= NSEQ; i++)
                c[i + m] ^= b[i];
            m++;
        }
    }
    memset(phi, 0, sizeof(*phi));
    for(int i = 0; i <= L; i++)
        if(c[i])
            phi->w[(L - i) >> 6] |= 1ull << ((L - i) & 63);
    return L;
}

static poly g_phi;

/* acc ^= src << shift (src: 3 words, acc: 6 words) */
static void xor_shifted(uint64_t* acc, const uint64_t* src, int shift)
{
    const int w = shift >> 6, s = shift & 63;
    for(int k = 0; k < 3; k++)
    {
        acc[w + k] ^= src[k] << s;
        if(s && w + k + 1 < 6)
            acc[w + k + 1] ^= src[k] >> (64 - s);
    }
}

/* a * b mod phi, a and b of degree < DEG */
static poly mulmod(const poly* a, const poly* b)
{
    poly acc;
    memset(&acc, 0, sizeof(acc));
    for(int i = 0; i < DEG; i++)
        if(getbit(a->w, i))
            xor_shifted(acc.w, b->w, i);
    for(int d = 2 * DEG - 2; d >= DEG; d--)
        if(getbit(acc.w, d))
            xor_shifted(acc.w, g_phi.w, d - DEG);
    return acc;
}

/* State p(A) s as window sums of the sequence of s. */
static void apply_poly(const poly* p, const uint32_t* s, uint32_t* out)
{
    uint32_t seq[SEQW];
    word_sequence(s, seq, SEQW);
    for(int j = 0; j < 5; j++)
        out[j] = 0;
    for(int k = 0; k < DEG; k++)
        if(getbit(p->w, k))
            for(int j = 0; j < 5; j++)
                out[j] ^= seq[k + j];
}

/* 160 x 160 GF(2) matrices: row r is the image of input bit r (word r / 32, bit r % 32). */
typedef struct
{
    uint32_t r[DEG][5];
} mat;

static void mat_apply(const mat* m, const uint32_t* x, uint32_t* y)
{
    uint32_t t[5] = {0, 0, 0, 0, 0};
    for(int r = 0; r < DEG; r++)
        if((x[r / 32] >> (r % 32)) & 1u)
            for(int k = 0; k < 5; k++)
                t[k] ^= m->r[r][k];
    memcpy(y, t, sizeof(t));
}

/* b after a */
static void mat_then(const mat* a, const mat* b, mat* out)
{
    mat t;
    for(int r = 0; r < DEG; r++)
        mat_apply(b, a->r[r], t.r[r]);
    *out = t;
}

static uint64_t g_rng = 0x9e3779b97f4a7c15ull;
static uint32_t rnd(void)
{
    g_rng ^= g_rng << 13;
    g_rng ^= g_rng >> 7;
    g_rng ^= g_rng << 17;
    return (uint32_t)(g_rng >> 16);
}

int main(int argc, char** argv)
{
    if(argc != 2)
    {
        fprintf(stderr, "usage: %s <output.bin>\n", argv[0]);
        return 2;
    }
    /* 1. phi from bit 0 of the word sequence of an arbitrary nonzero state */
    {
        const uint32_t s0[5] = {123456789u, 362436069u, 521288629u, 88675123u, 5783321u};
        uint32_t       seq[NSEQ];
        int            bits[NSEQ];
        word_sequence(s0, seq, NSEQ);
        for(int n = 0; n < NSEQ; n++)
            bits[n] = (int)(seq[n] & 1u);
        const int L = berlekamp_massey(bits, &g_phi);
        if(L != DEG)
        {
            fprintf(stderr, "characteristic polynomial of degree %d, expected %d\n", L, DEG);
            return 1;
        }
    }
    /* 2. q = x^(2^67) mod phi */
    poly q;
    memset(&q, 0, sizeof(q));
    q.w[0] = 2; /* x */
    for(int i = 0; i < 67; i++)
        q = mulmod(&q, &q);
    /* 3. p_e = q^e */
    uint32_t* out = calloc((size_t)5 * ENGINES, sizeof(uint32_t));
    poly*     keep = calloc(ENGINES, sizeof(poly));
    if(!out || !keep)
        return 1;
    poly p;
    memset(&p, 0, sizeof(p));
    p.w[0] = 1;
    for(int e = 0; e < ENGINES; e++)
    {
        keep[e] = p;
        for(int j = 0; j < 5; j++)
            out[(size_t)j * ENGINES + e] = (uint32_t)(p.w[j / 2] >> (32 * (j & 1)));
        p = mulmod(&p, &q);
    }
    /* 4. self-check against matrix powers of the one-step map */
    {
        mat a;
        for(int r = 0; r < DEG; r++)
        {
            uint32_t x[5] = {0, 0, 0, 0, 0};
            x[r / 32]     = 1u << (r % 32);
            xorwow_step(x);
            memcpy(a.r[r], x, sizeof(x));
        }
        mat j = a; /* A^(2^67) */
        for(int i = 0; i < 67; i++)
            mat_then(&j, &j, &j);
        const int checks[] = {0, 1, 2, 3, 5, 64, 1000, 65537, ENGINES - 1};
        for(size_t c = 0; c < sizeof(checks) / sizeof(checks[0]); c++)
        {
            const int e    = checks[c];
            uint32_t  s[5] = {rnd(), rnd(), rnd(), rnd(), rnd()};
            uint32_t  want[5], got[5];
            /* J^e s by binary powers */
            mat pw = j;
            memcpy(want, s, sizeof(s));
            for(int b = e; b; b >>= 1)
            {
                if(b & 1)
                    mat_apply(&pw, want, want);
                if(b > 1)
                    mat_then(&pw, &pw, &pw);
            }
            apply_poly(&keep[e], s, got);
            if(memcmp(want, got, sizeof(got)) != 0)
            {
                fprintf(stderr, "jump polynomial of engine %d does not match the matrix jump\n", e);
                return 1;
            }
        }
    }
    FILE* f = fopen(argv[1], "wb");
    if(!f)
        return 1;
    if(fwrite(out, sizeof(uint32_t), (size_t)5 * ENGINES, f) != (size_t)5 * ENGINES)
        return 1;
    fclose(f);
    free(out);
    free(keep);
    return 0;
}
