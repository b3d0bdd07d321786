// make_device_jump_tables.cpp -- writes include/rocrand/rocrand_b200_jump_tables.h, the
// skip-ahead matrices of the device API's MRG32k3a and MRG31k3p states.
//
// The device API (rocrand_kernel.h) advances an MRG state by `offset` values, `subsequence`
// subsequences or `sequence` sequences by binary powers of the one-step matrices:
//   offset:      A^(2^k),            k = 0..63
//   subsequence: A^(2^(S+k)),        S = 76 (MRG32k3a, rocrand_mrg32k3a.h:125-141) or
//                                    72 (MRG31k3p, rocrand_mrg31k3p.h:115-133)
//   sequence:    A^(2^(Q+k)),        Q = 127 (MRG32k3a) or 134 (MRG31k3p)
// for both components.  The matrices are computed here from the recurrences
// (rocrand_b200/csrc/jump_tables.cpp) by repeated squaring, so they are exact by
// construction; a user kernel gets them as __device__ arrays.
//
// Usage: make_device_jump_tables <output.h>
#include "../csrc/jump_tables.hpp"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

using namespace rb200;

// ---- XORWOW jump polynomials -------------------------------------------------------------
// The xorshift part of XORWOW is a linear bijection A on 160 bits with characteristic
// polynomial phi (degree 160), so A^N s = (x^N mod phi)(A) s, and A^k s is the state after k
// steps.  The device API stores q = x^(d 4^i) mod phi (offsets) and x^(d 4^i 2^67) mod phi
// (subsequences), i < 32, d = 1..3, 5 words each, and applies them by stepping a copy of the
// state 160 times and XOR-ing the states at the set coefficients.

namespace
{

struct Poly
{
    uint64_t w[6] = {0, 0, 0, 0, 0, 0};
};

int bit(const uint64_t* a, int i)
{
    return static_cast<int>((a[i >> 6] >> (i & 63)) & 1u);
}

void xor_shifted(uint64_t* acc, const uint64_t* src, int shift)
{
    const int w = shift >> 6, s = shift & 63;
    for(int k = 0; k < 3; k++)
    {
        acc[w + k] ^= src[k] << s;
        if(s && w + k + 1 < 6)
            acc[w + k + 1] ^= src[k] >> (64 - s);
    }
}

Poly g_phi;

Poly mulmod(const Poly& a, const Poly& b)
{
    Poly acc;
    for(int i = 0; i < 160; i++)
        if(bit(a.w, i))
            xor_shifted(acc.w, b.w, i);
    for(int d = 318; d >= 160; d--)
        if(bit(acc.w, d))
            xor_shifted(acc.w, g_phi.w, d - 160);
    return acc;
}

void xorwow_step(uint32_t* x)
{
    const uint32_t t = x[0] ^ (x[0] >> 2);
    x[0]             = x[1];
    x[1]             = x[2];
    x[2]             = x[3];
    x[3]             = x[4];
    x[4]             = (x[4] ^ (x[4] << 4)) ^ (t ^ (t << 1));
}

// phi by Berlekamp-Massey over bit 0 of 2 * 160 + 64 outputs of the word sequence
bool xorwow_phi()
{
    const int        n = 384;
    uint32_t         x[5] = {123456789u, 362436069u, 521288629u, 88675123u, 5783321u};
    std::vector<int> s(n), c(n + 1, 0), b(n + 1, 0), t;
    for(int i = 0; i < n; i++)
    {
        xorwow_step(x);
        s[i] = static_cast<int>(x[4] & 1u);
    }
    c[0] = b[0] = 1;
    int L = 0, m = 1;
    for(int i = 0; i < n; i++)
    {
        int d = s[i];
        for(int j = 1; j <= L; j++)
            d ^= c[j] & s[i - j];
        if(!d)
        {
            m++;
            continue;
        }
        t = c;
        for(int j = 0; j + m <= n; j++)
            c[j + m] ^= b[j];
        if(2 * L <= i)
        {
            L = i + 1 - L;
            b = t;
            m = 1;
        }
        else
        {
            m++;
        }
    }
    if(L != 160)
        return false;
    for(int i = 0; i <= L; i++)
        if(c[i])
            g_phi.w[(L - i) >> 6] |= 1ull << ((L - i) & 63);
    return true;
}

Poly x_pow2(int k) // x^(2^k) mod phi
{
    Poly p;
    p.w[0] = 2;
    for(int i = 0; i < k; i++)
        p = mulmod(p, p);
    return p;
}

// check q(A) s == A^n s on a state for small n
bool check(const Poly& q, unsigned n)
{
    uint32_t s[5] = {0x12345678u, 0x9abcdef0u, 0x0badf00du, 0xdeadbeefu, 0x13579bdfu}, y[5] = {0, 0, 0, 0, 0};
    uint32_t x[5];
    std::memcpy(x, s, sizeof(x));
    for(int k = 0; k < 160; k++)
    {
        if(bit(q.w, k))
            for(int j = 0; j < 5; j++)
                y[j] ^= x[j];
        xorwow_step(x);
    }
    std::memcpy(x, s, sizeof(x));
    for(unsigned i = 0; i < n; i++)
        xorwow_step(x);
    return std::memcmp(x, y, sizeof(x)) == 0;
}

void emit_xorwow(FILE* f, const char* name, int first)
{
    Poly base = x_pow2(first); // x^(2^first)
    for(int copy = 0; copy < 2; copy++)
    {
        std::fprintf(f, "%s const unsigned int %s_%s[32 * 3 * 5] = {\n", copy == 0 ? "static __device__" : "static",
                     name, copy == 0 ? "d" : "h");
        Poly digit = base; // x^(4^i 2^first)
        for(int i = 0; i < 32; i++)
        {
            Poly p = digit;
            for(int d = 1; d <= 3; d++)
            {
                std::fprintf(f, "   ");
                for(int j = 0; j < 5; j++)
                    std::fprintf(f, " %uu,", static_cast<unsigned>(p.w[j / 2] >> (32 * (j & 1))));
                std::fprintf(f, "\n");
                p = mulmod(p, digit);
            }
            digit = mulmod(digit, digit);
            digit = mulmod(digit, digit);
        }
        std::fprintf(f, "};\n");
    }
}

// ---- LFSR113 jump polynomials --------------------------------------------------------------
// Each of the four Tausworthe components is linear on its 32-bit word, but its step ignores
// the word's low bits (they are masked off), so on the whole word the step T is not
// invertible; on its image V (dimension k = 31, 29, 28, 25) it is, with a primitive minimal
// polynomial phi of degree k.  Hence T^N z = T^(N-1) (T z) = (x^(N-1) mod phi)(T) (T z) for
// N >= 1 and any word z.  The device API stores x^(d 4^i S - 1) mod phi per component
// (S = 1 for offsets, 2^55 for subsequences), i < 32, d = 1..3, one word each.

uint32_t lfsr_step(int j, uint32_t z)
{
    uint32_t b;
    switch(j)
    {
        case 0: b = ((z << 6) ^ z) >> 13; return ((z & 4294967294u) << 18) ^ b;
        case 1: b = ((z << 2) ^ z) >> 27; return ((z & 4294967288u) << 2) ^ b;
        case 2: b = ((z << 13) ^ z) >> 21; return ((z & 4294967280u) << 7) ^ b;
        default: b = ((z << 3) ^ z) >> 12; return ((z & 4294967168u) << 13) ^ b;
    }
}

struct SmallField
{
    uint64_t phi = 0; // minimal polynomial (bit k = coefficient of x^k)
    int      deg = 0;
    uint64_t mulmod(uint64_t a, uint64_t b) const
    {
        uint64_t acc = 0;
        for(int i = 0; i < deg; i++)
            if((a >> i) & 1u)
                acc ^= b << i;
        for(int d = 2 * deg - 2; d >= deg; d--)
            if((acc >> d) & 1u)
                acc ^= phi << (d - deg);
        return acc;
    }
};

bool lfsr_field(int j, SmallField& f)
{
    const int        n = 96;
    uint32_t         z = lfsr_step(j, 0x9e3779b9u);
    std::vector<int> s(n), c(n + 1, 0), b(n + 1, 0), t;
    for(int i = 0; i < n; i++)
    {
        s[i] = static_cast<int>(z >> 31);
        z    = lfsr_step(j, z);
    }
    c[0] = b[0] = 1;
    int L = 0, m = 1;
    for(int i = 0; i < n; i++)
    {
        int d = s[i];
        for(int k = 1; k <= L; k++)
            d ^= c[k] & s[i - k];
        if(!d)
        {
            m++;
            continue;
        }
        t = c;
        for(int k = 0; k + m <= n; k++)
            c[k + m] ^= b[k];
        if(2 * L <= i)
        {
            L = i + 1 - L;
            b = t;
            m = 1;
        }
        else
        {
            m++;
        }
    }
    const int want[4] = {31, 29, 28, 25};
    if(L != want[j])
        return false;
    f.deg = L;
    f.phi = 0;
    for(int i = 0; i <= L; i++)
        if(c[i])
            f.phi |= 1ull << (L - i);
    return (f.phi & 1u) != 0;
}

// T^N z by the stored polynomial q = x^(N-1) mod phi
uint32_t lfsr_apply(int j, const SmallField& f, uint64_t q, uint32_t z)
{
    uint32_t y = lfsr_step(j, z), acc = 0;
    for(int k = 0; k < f.deg; k++)
    {
        if((q >> k) & 1u)
            acc ^= y;
        y = lfsr_step(j, y);
    }
    return acc;
}

int emit_lfsr113(FILE* f)
{
    SmallField fld[4];
    for(int j = 0; j < 4; j++)
        if(!lfsr_field(j, fld[j]))
            return 1;
    const int  firsts[2] = {0, 55};
    const char* names[2] = {"lfsr113_poly", "lfsr113_poly_sub"};
    const Gf2Matrix a    = lfsr113_step_matrix();
    for(int kind = 0; kind < 2; kind++)
    {
        // value[i][d-1][j]
        std::vector<uint32_t> v(32 * 3 * 4);
        for(int j = 0; j < 4; j++)
        {
            const SmallField& F   = fld[j];
            const uint64_t    inv = F.phi >> 1; // x^-1 = (phi - 1) / x
            uint64_t          dig = 2;           // x
            for(int k = 0; k < firsts[kind]; k++)
                dig = F.mulmod(dig, dig);        // x^(2^first)
            for(int i = 0; i < 32; i++)
            {
                uint64_t p = dig;
                for(int d = 1; d <= 3; d++)
                {
                    v[(i * 3 + (d - 1)) * 4 + j] = static_cast<uint32_t>(F.mulmod(p, inv));
                    p                            = F.mulmod(p, dig);
                }
                dig = F.mulmod(dig, dig);
                dig = F.mulmod(dig, dig);
            }
        }
        // self-check on two digits against the 128-bit step matrix raised to the jump
        for(int i : {0, 1, 3})
        {
            for(int d = 1; d <= 3; d++)
            {
                const unsigned long long e  = static_cast<unsigned long long>(d) << (2 * i);
                Gf2Matrix                m  = gf2_pow(kind == 0 ? a : gf2_pow2(a, 55), e);
                uint32_t                 z[4] = {0x12345679u, 0xfedcba98u, 0x0f0f0f0fu, 0xc0ffee11u}, w[4];
                m.apply(z, w);
                for(int j = 0; j < 4; j++)
                    if(lfsr_apply(j, fld[j], v[(i * 3 + (d - 1)) * 4 + j], z[j]) != w[j])
                        return 1;
            }
        }
        for(int copy = 0; copy < 2; copy++)
        {
            std::fprintf(f, "%s const unsigned int %s_%s[32 * 3 * 4] = {\n",
                         copy == 0 ? "static __device__" : "static", names[kind], copy == 0 ? "d" : "h");
            for(int r = 0; r < 32 * 3; r++)
                std::fprintf(f, "    %uu, %uu, %uu, %uu,\n", v[r * 4], v[r * 4 + 1], v[r * 4 + 2], v[r * 4 + 3]);
            std::fprintf(f, "};\n");
        }
    }
    std::fprintf(f, "static __device__ const unsigned int lfsr113_degree_d[4] = {%d, %d, %d, %d};\n"
                    "static const unsigned int lfsr113_degree_h[4] = {%d, %d, %d, %d};\n",
                 fld[0].deg, fld[1].deg, fld[2].deg, fld[3].deg, fld[0].deg, fld[1].deg, fld[2].deg, fld[3].deg);
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    if(argc != 2)
        return 2;
    FILE* f = std::fopen(argv[1], "w");
    if(!f)
        return 1;
    std::fprintf(f,
                 "/* Generated by rocrand_b200/data/make_device_jump_tables.cpp: do not edit.\n"
                 " * Skip-ahead matrices of the device API's MRG states (rocrand_kernel.h): 64\n"
                 " * row-major 3x3 matrices per table, entry k = A^(2^(first + k)) of one\n"
                 " * component.  Each table has a device copy (_d) and a host copy (_h). */\n"
                 "#ifndef ROCRAND_B200_JUMP_TABLES_H_\n#define ROCRAND_B200_JUMP_TABLES_H_\n\n"
                 "namespace rocrand_b200_detail\n{\n\n");
    struct T
    {
        const char* name;
        const char* type;
        ModMatrix   a;
        int         first;
    } tabs[] = {
        {"mrg32k3a_a1", "unsigned long long", mrg32k3a_step1(), 0},
        {"mrg32k3a_a2", "unsigned long long", mrg32k3a_step2(), 0},
        {"mrg32k3a_a1_sub", "unsigned long long", mrg32k3a_step1(), 76},
        {"mrg32k3a_a2_sub", "unsigned long long", mrg32k3a_step2(), 76},
        {"mrg32k3a_a1_seq", "unsigned long long", mrg32k3a_step1(), 127},
        {"mrg32k3a_a2_seq", "unsigned long long", mrg32k3a_step2(), 127},
        {"mrg31k3p_a1", "unsigned int", mrg31k3p_step1(), 0},
        {"mrg31k3p_a2", "unsigned int", mrg31k3p_step2(), 0},
        {"mrg31k3p_a1_sub", "unsigned int", mrg31k3p_step1(), 72},
        {"mrg31k3p_a2_sub", "unsigned int", mrg31k3p_step2(), 72},
        {"mrg31k3p_a1_seq", "unsigned int", mrg31k3p_step1(), 134},
        {"mrg31k3p_a2_seq", "unsigned int", mrg31k3p_step2(), 134},
    };
    for(const T& t : tabs)
    {
        for(int copy = 0; copy < 2; copy++)
        {
            ModMatrix a = mod_pow2(t.a, t.first);
            std::fprintf(f, "%s const %s %s_%s[64 * 9] = {\n",
                         copy == 0 ? "static __device__" : "static", t.type, t.name, copy == 0 ? "d" : "h");
            for(int k = 0; k < 64; k++)
            {
                std::fprintf(f, "   ");
                for(int i = 0; i < 9; i++)
                    std::fprintf(f, " %lluu,", static_cast<unsigned long long>(a.a[i]));
                std::fprintf(f, "\n");
                a = a.mul(a);
            }
            std::fprintf(f, "};\n");
        }
    }
    if(!xorwow_phi())
        return 1;
    // self-check: the offset digits 1..3 of position 0 are x, x^2, x^3
    {
        Poly q = x_pow2(0);
        if(!check(q, 1) || !check(mulmod(q, q), 2) || !check(mulmod(mulmod(q, q), q), 3))
            return 1;
    }
    std::fprintf(f, "/* XORWOW: x^(d 4^i) and x^(d 4^i 2^67) modulo the characteristic polynomial of the\n"
                    " * xorshift step, i < 32, d = 1..3, 5 words each (bit k = coefficient of x^k). */\n");
    emit_xorwow(f, "xorwow_poly", 0);
    emit_xorwow(f, "xorwow_poly_sub", 67);
    std::fprintf(f, "/* LFSR113: per component, x^(d 4^i S - 1) modulo its minimal polynomial on the image of\n"
                    " * its step (S = 1 or 2^55), i < 32, d = 1..3, words [i][d-1][component]. */\n");
    if(emit_lfsr113(f) != 0)
        return 1;
    std::fprintf(f, "\n} // namespace rocrand_b200_detail\n\n#endif\n");
    std::fclose(f);
    return 0;
}
