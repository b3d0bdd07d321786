// jump_tables.hpp -- skip-ahead matrices of the stateful engines, computed on the host.
//
// XORWOW (160-bit xorshift part) and LFSR113 (4 x 32-bit Tausworthe) are linear maps over
// GF(2); MRG32k3a and MRG31k3p are two 3x3 recurrences modulo m1 / m2.  A jump by k steps
// is the k-th power of the one-step matrix.  The reference ships precomputed tables
// (rocrand_{xorwow,lfsr113,mrg32k3a,mrg31k3p}_precomputed.h); here the one-step matrix is
// built from the engine's own recurrence and raised to the needed powers by squaring, so
// the tables are exact by construction and need no data files.
//
// Layouts (device copies are uploaded once per device):
//  * GF(2) matrix of an N-word state: N*32 rows of N words; row r is the image of input bit
//    r (word r/32, bit r%32), so y = XOR of the rows of the set bits of x.
//  * mod-m matrix: 3x3 row-major, entries reduced to [0, m).
#pragma once

#include <cstdint>
#include <vector>

namespace rb200
{

// Square GF(2) matrix over a state of N 32-bit words.
struct Gf2Matrix
{
    int                   words = 0; // N
    std::vector<uint32_t> rows;      // (N*32) x N
    explicit Gf2Matrix(int n = 0) : words(n), rows(static_cast<size_t>(n) * 32 * n, 0u) {}
    static Gf2Matrix identity(int n);
    void             apply(const uint32_t* x, uint32_t* y) const; // y = M x
    Gf2Matrix        then(const Gf2Matrix& b) const;               // b after this: x -> b(M x)
};

// The one-step maps of the GF(2) engines.
Gf2Matrix xorwow_step_matrix();  // 5 words: x[0..4] (xorshift part, rocrand_xorwow.h:165-177)
Gf2Matrix lfsr113_step_matrix(); // 4 words: z.x, z.y, z.z, z.w (rocrand_lfsr113.h:146-160)

// M^(2^k) by k squarings.
Gf2Matrix gf2_pow2(const Gf2Matrix& m, int k);
// M^e for a 64-bit exponent.
Gf2Matrix gf2_pow(const Gf2Matrix& m, unsigned long long e);

// 3x3 matrix modulo m.
struct ModMatrix
{
    uint64_t m = 0;
    uint64_t a[9] = {};
    static ModMatrix identity(uint64_t mod);
    void             apply(const uint32_t* x, uint32_t* y) const; // y = A x mod m (x as integers)
    ModMatrix        mul(const ModMatrix& b) const;               // this * b
};

ModMatrix mod_pow2(const ModMatrix& a, int k);
ModMatrix mod_pow(const ModMatrix& a, unsigned long long e);

// One-step matrices of the MRG components (state order: oldest..newest as the engine keeps it).
ModMatrix mrg32k3a_step1();
ModMatrix mrg32k3a_step2();
ModMatrix mrg31k3p_step1();
ModMatrix mrg31k3p_step2();

// Per-digit jump tables for the engine (subsequence) skip of the device init kernel:
// for digit position p (radix 4) and digit value d in 1..3, J^(d * 4^p) where J is the
// subsequence stride; positions 0..8 cover engine ids below 2^18.
constexpr int kJumpDigits = 9;
std::vector<uint32_t> gf2_digit_tables(const Gf2Matrix& j);       // [p][d-1] matrices
std::vector<uint64_t> mod_digit_tables(const ModMatrix& j1, const ModMatrix& j2); // [p][d-1][c]

} // namespace rb200
