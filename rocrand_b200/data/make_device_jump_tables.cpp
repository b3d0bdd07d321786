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
    std::fprintf(f, "\n} // namespace rocrand_b200_detail\n\n#endif\n");
    std::fclose(f);
    return 0;
}
