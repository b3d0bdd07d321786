// jump_tables.cpp -- skip-ahead matrices of the stateful engines (see jump_tables.hpp).
#include "jump_tables.hpp"

#include <cstring>

namespace rb200
{

Gf2Matrix Gf2Matrix::identity(int n)
{
    Gf2Matrix m(n);
    for(int r = 0; r < n * 32; r++)
        m.rows[static_cast<size_t>(r) * n + r / 32] = 1u << (r % 32);
    return m;
}

void Gf2Matrix::apply(const uint32_t* x, uint32_t* y) const
{
    for(int k = 0; k < words; k++)
        y[k] = 0;
    for(int r = 0; r < words * 32; r++)
        if((x[r / 32] >> (r % 32)) & 1u)
            for(int k = 0; k < words; k++)
                y[k] ^= rows[static_cast<size_t>(r) * words + k];
}

Gf2Matrix Gf2Matrix::then(const Gf2Matrix& b) const
{
    Gf2Matrix c(words);
    for(int r = 0; r < words * 32; r++)
        b.apply(&rows[static_cast<size_t>(r) * words], &c.rows[static_cast<size_t>(r) * words]);
    return c;
}

// Builds the matrix of a linear one-step map by applying it to every basis vector.
template<class Step>
static Gf2Matrix probe(int n, Step step)
{
    Gf2Matrix m(n);
    std::vector<uint32_t> x(n);
    for(int r = 0; r < n * 32; r++)
    {
        std::fill(x.begin(), x.end(), 0u);
        x[r / 32] = 1u << (r % 32);
        step(x.data());
        std::memcpy(&m.rows[static_cast<size_t>(r) * n], x.data(), sizeof(uint32_t) * n);
    }
    return m;
}

Gf2Matrix xorwow_step_matrix()
{
    // xorshift160 part of the XORWOW step (the Weyl counter is added separately).
    return probe(5, [](uint32_t* x) {
        const uint32_t t = x[0] ^ (x[0] >> 2);
        x[0]             = x[1];
        x[1]             = x[2];
        x[2]             = x[3];
        x[3]             = x[4];
        x[4]             = (x[4] ^ (x[4] << 4)) ^ (t ^ (t << 1));
    });
}

Gf2Matrix lfsr113_step_matrix()
{
    // The four Tausworthe components (L'Ecuyer's LFSR113 parameters).
    return probe(4, [](uint32_t* z) {
        uint32_t b;
        b    = ((z[0] << 6) ^ z[0]) >> 13;
        z[0] = ((z[0] & 4294967294u) << 18) ^ b;
        b    = ((z[1] << 2) ^ z[1]) >> 27;
        z[1] = ((z[1] & 4294967288u) << 2) ^ b;
        b    = ((z[2] << 13) ^ z[2]) >> 21;
        z[2] = ((z[2] & 4294967280u) << 7) ^ b;
        b    = ((z[3] << 3) ^ z[3]) >> 12;
        z[3] = ((z[3] & 4294967168u) << 13) ^ b;
    });
}

Gf2Matrix gf2_pow2(const Gf2Matrix& m, int k)
{
    Gf2Matrix p = m;
    for(int i = 0; i < k; i++)
        p = p.then(p);
    return p;
}

Gf2Matrix gf2_pow(const Gf2Matrix& m, unsigned long long e)
{
    Gf2Matrix r = Gf2Matrix::identity(m.words);
    Gf2Matrix p = m;
    while(e)
    {
        if(e & 1)
            r = r.then(p);
        e >>= 1;
        if(e)
            p = p.then(p);
    }
    return r;
}

ModMatrix ModMatrix::identity(uint64_t mod)
{
    ModMatrix i;
    i.m    = mod;
    i.a[0] = i.a[4] = i.a[8] = 1;
    return i;
}

void ModMatrix::apply(const uint32_t* x, uint32_t* y) const
{
    for(int r = 0; r < 3; r++)
    {
        unsigned __int128 s = 0;
        for(int c = 0; c < 3; c++)
            s += static_cast<unsigned __int128>(a[r * 3 + c]) * x[c];
        y[r] = static_cast<uint32_t>(s % m);
    }
}

ModMatrix ModMatrix::mul(const ModMatrix& b) const
{
    ModMatrix c;
    c.m = m;
    for(int r = 0; r < 3; r++)
        for(int k = 0; k < 3; k++)
        {
            unsigned __int128 s = 0;
            for(int j = 0; j < 3; j++)
                s += static_cast<unsigned __int128>(a[r * 3 + j]) * b.a[j * 3 + k];
            c.a[r * 3 + k] = static_cast<uint64_t>(s % m);
        }
    return c;
}

ModMatrix mod_pow2(const ModMatrix& a, int k)
{
    ModMatrix p = a;
    for(int i = 0; i < k; i++)
        p = p.mul(p);
    return p;
}

ModMatrix mod_pow(const ModMatrix& a, unsigned long long e)
{
    ModMatrix r = ModMatrix::identity(a.m);
    ModMatrix p = a;
    while(e)
    {
        if(e & 1)
            r = p.mul(r);
        e >>= 1;
        if(e)
            p = p.mul(p);
    }
    return r;
}

// MRG32k3a (L'Ecuyer 1999): x1_n = 1403580 x1_{n-2} - 810728 x1_{n-3} mod m1,
// x2_n = 527612 x2_{n-1} - 1370589 x2_{n-3} mod m2; state (x_{n-3}, x_{n-2}, x_{n-1}).
ModMatrix mrg32k3a_step1()
{
    const uint64_t m1 = 4294967087ull;
    ModMatrix      a;
    a.m  = m1;
    a.a[1] = 1;
    a.a[5] = 1;
    a.a[6] = m1 - 810728;
    a.a[7] = 1403580;
    return a;
}

ModMatrix mrg32k3a_step2()
{
    const uint64_t m2 = 4294944443ull;
    ModMatrix      a;
    a.m  = m2;
    a.a[1] = 1;
    a.a[5] = 1;
    a.a[6] = m2 - 1370589;
    a.a[8] = 527612;
    return a;
}

// MRG31k3p (L'Ecuyer & Touzin 2000): x1_n = 2^22 x1_{n-2} + (2^7+1) x1_{n-3} mod m1,
// x2_n = 2^15 x2_{n-1} + (2^15+1) x2_{n-3} mod m2; state (x_{n-1}, x_{n-2}, x_{n-3}).
ModMatrix mrg31k3p_step1()
{
    ModMatrix a;
    a.m    = 2147483647ull;
    a.a[1] = 1u << 22;
    a.a[2] = (1u << 7) + 1;
    a.a[3] = 1;
    a.a[7] = 1;
    return a;
}

ModMatrix mrg31k3p_step2()
{
    ModMatrix a;
    a.m    = 2147462579ull;
    a.a[0] = 1u << 15;
    a.a[2] = (1u << 15) + 1;
    a.a[3] = 1;
    a.a[7] = 1;
    return a;
}

std::vector<uint32_t> gf2_digit_tables(const Gf2Matrix& j)
{
    const size_t          msize = j.rows.size();
    std::vector<uint32_t> out(static_cast<size_t>(kJumpDigits) * 3 * msize);
    Gf2Matrix             base = j; // J^(4^p)
    for(int p = 0; p < kJumpDigits; p++)
    {
        Gf2Matrix acc = base;
        for(int d = 1; d <= 3; d++)
        {
            std::memcpy(&out[(static_cast<size_t>(p) * 3 + (d - 1)) * msize], acc.rows.data(),
                        msize * sizeof(uint32_t));
            if(d < 3)
                acc = acc.then(base);
        }
        base = gf2_pow2(base, 2);
    }
    return out;
}

std::vector<uint64_t> mod_digit_tables(const ModMatrix& j1, const ModMatrix& j2)
{
    std::vector<uint64_t> out(static_cast<size_t>(kJumpDigits) * 3 * 2 * 9);
    ModMatrix             b1 = j1, b2 = j2;
    for(int p = 0; p < kJumpDigits; p++)
    {
        ModMatrix a1 = b1, a2 = b2;
        for(int d = 1; d <= 3; d++)
        {
            uint64_t* dst = &out[((static_cast<size_t>(p) * 3 + (d - 1)) * 2) * 9];
            std::memcpy(dst, a1.a, sizeof(a1.a));
            std::memcpy(dst + 9, a2.a, sizeof(a2.a));
            if(d < 3)
            {
                a1 = a1.mul(b1);
                a2 = a2.mul(b2);
            }
        }
        b1 = mod_pow2(b1, 2);
        b2 = mod_pow2(b2, 2);
    }
    return out;
}

} // namespace rb200
