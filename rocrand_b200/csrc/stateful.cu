// stateful.cu -- XORWOW, MRG32k3a, MRG31k3p and LFSR113 generators.
//
// Output contract of the reference (xorwow.hpp:63-161, mrg.hpp:66-157, lfsr113.hpp:66-160),
// all on E = 131072 persistent engines (512 x 256, config_defaults.hpp:33-66):
//   * engine e starts as Engine(seed, subsequence = e, offset / E + (e < start)) with
//     start = offset % E (xorwow.hpp:45-61, 295);
//   * output vector j (ow elements) is the next application of the distribution on engine
//     (j + start) % E -- i.e. "slot" t = j % E drives engine (t + start) % E and writes
//     vectors t, t + E, t + 2E, ...;
//   * with ow > 1, the slot t == vec_n % E then writes the misaligned head, and then the
//     tail, from the same engine (xorwow.hpp:121-157);
//   * afterwards start += ceil(n / ow) mod E (xorwow.hpp:385-389).
//
// B200 layout: engine states live in HBM as a structure of arrays (word w of engine e at
// arena[w * E + e]) so every load/store of a warp is coalesced; a thread owns one slot,
// keeps its engine in registers for the whole call and writes it back only if it advanced.
// Initialisation is split: the host applies the common offset jump to the seeded state
// once (two base states: offset/E and offset/E + 1), the device applies each engine's
// subsequence jump J^e: from per-digit tables (jump_tables.hpp), at most 9 matrix-vector
// products per engine, for MRG32k3a, MRG31k3p and LFSR113; by jump polynomial for XORWOW
// (stateful_engines.cuh: 40 shared-memory table reads per engine).
#include "common.hpp"
#include "dist.cuh"
#include "generators.hpp"
#include "host_exec.hpp"
#include "jump_tables.hpp"
#include "launch.cuh"
#include "poisson.hpp"
#include "stateful_engines.cuh"
#include "batch.hpp"

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>
#include <vector>

extern "C" const unsigned char rb200_xorwow_jump_begin[];
extern "C" const unsigned char rb200_xorwow_jump_end[];

namespace rb200
{

constexpr uint32_t kE = kStatefulEngines; // 131072

struct InitArgs
{
    uint32_t base[2][6]; // [0]: offset/E, [1]: offset/E + 1 (engines below start)
    uint32_t start;
    uint32_t* arena;
};

// x <- J^e x from the per-digit tables: one matrix per non-zero base-4 digit of e (GF(2)
// engines; the device init kernel and the CPU path share it).
template<int NJ>
__host__ __device__ __forceinline__ void gf2_jump_digits(const uint32_t* tables, uint32_t e, uint32_t* x)
{
    constexpr size_t msize = static_cast<size_t>(NJ) * 32 * NJ;
    for(int p = 0; p < kJumpDigits; p++)
    {
        const uint32_t d = (e >> (2 * p)) & 3u;
        if(d)
            gf2_apply<NJ>(tables + (static_cast<size_t>(p) * 3 + (d - 1)) * msize, x);
    }
}

// The same for the MRG engines: each digit matrix is a pair (component 1 mod m1, component
// 2 mod m2) of 3 x 3 matrices.
__host__ __device__ __forceinline__ void mod_jump_digits(const uint64_t* tables, uint64_t m1, uint64_t m2,
                                                         uint32_t e, uint32_t* x)
{
    for(int p = 0; p < kJumpDigits; p++)
    {
        const uint32_t d = (e >> (2 * p)) & 3u;
        if(d)
        {
            const uint64_t* t = tables + ((static_cast<size_t>(p) * 3 + (d - 1)) * 2) * 9;
            mod_apply(t, m1, x);
            mod_apply(t + 9, m2, x + 3);
        }
    }
}

// GF(2) engines (XORWOW: 5 jump words + the Weyl counter copied; LFSR113: 4 words).
template<int NJ, int NW>
__global__ void __launch_bounds__(kBlock) init_gf2(InitArgs a, const uint32_t* __restrict__ tables)
{
    const uint32_t e = blockIdx.x * kBlock + threadIdx.x;
    if(e >= kE)
        return;
    uint32_t x[NW];
    const int which = e < a.start ? 1 : 0;
#pragma unroll
    for(int k = 0; k < NW; k++)
        x[k] = a.base[which][k];
    gf2_jump_digits<NJ>(tables, e, x);
#pragma unroll
    for(int k = 0; k < NW; k++)
        a.arena[static_cast<size_t>(k) * kE + e] = x[k];
}

// XORWOW engines by jump polynomial: each block builds the window tables of the base(s)
// its engines use in shared memory, then each thread seeds kXorwowInitPerThread engines.
constexpr uint32_t kXorwowInitPerThread = 2;

struct XorwowInitArgs
{
    InitArgs a;
    uint32_t seq[2][kXorwowSeqWords]; // word sequences of base[0] and base[1]
};

__global__ void __launch_bounds__(kBlock)
    init_xorwow(const __grid_constant__ XorwowInitArgs a, const uint32_t* __restrict__ polys)
{
    __shared__ XorwowJumpTable table[2];
    __shared__ uint32_t        seq[2][kXorwowSeqWords];
    constexpr uint32_t         per_block = kBlock * kXorwowInitPerThread;
    const uint32_t             e0        = blockIdx.x * per_block; // kE is a multiple of it
    const bool                 need1     = e0 < a.a.start;         // engines below start
    const bool                 need0     = e0 + per_block > a.a.start;
    for(uint32_t i = threadIdx.x; i < 2 * kXorwowSeqWords; i += kBlock)
        seq[i / kXorwowSeqWords][i % kXorwowSeqWords] = a.seq[i / kXorwowSeqWords][i % kXorwowSeqWords];
    __syncthreads();
    if(need0)
        xorwow_build_jump_table(table[0], seq[0], threadIdx.x, kBlock);
    if(need1)
        xorwow_build_jump_table(table[1], seq[1], threadIdx.x, kBlock);
    __syncthreads();
#pragma unroll
    for(uint32_t k = 0; k < kXorwowInitPerThread; k++)
    {
        const uint32_t e     = e0 + k * kBlock + threadIdx.x;
        const int      which = e < a.a.start ? 1 : 0;
        uint32_t       x[5];
        xorwow_jump(table[which], polys, e, x);
#pragma unroll
        for(int w = 0; w < 5; w++)
            a.a.arena[static_cast<size_t>(w) * kE + e] = x[w];
        a.a.arena[static_cast<size_t>(5) * kE + e] = a.a.base[which][5];
    }
}

// MRG engines: two 3-word components modulo m1 and m2.
__global__ void __launch_bounds__(kBlock)
    init_mrg(InitArgs a, const uint64_t* __restrict__ tables, uint64_t m1, uint64_t m2)
{
    const uint32_t e = blockIdx.x * kBlock + threadIdx.x;
    if(e >= kE)
        return;
    uint32_t  x[6];
    const int which = e < a.start ? 1 : 0;
#pragma unroll
    for(int k = 0; k < 6; k++)
        x[k] = a.base[which][k];
    mod_jump_digits(tables, m1, m2, e, x);
#pragma unroll
    for(int k = 0; k < 6; k++)
        a.arena[static_cast<size_t>(k) * kE + e] = x[k];
}

// ---- generation ----

struct FillArgs
{
    uint32_t*          arena;
    uint32_t           start;
    uint32_t           head, tail;
    unsigned char*     data;
    unsigned char*     vec;
    unsigned long long n, vec_n;
};

template<class E, class F>
__global__ void __launch_bounds__(kBlock) stateful_fill(FillArgs a, F f)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const F g = stage_table(f, smem);

    const uint32_t t = blockIdx.x * kBlock + threadIdx.x; // slot
    if(t >= kE)
        return;
    const bool loops = t < a.vec_n;
    const bool edges = F::ow > 1 && (a.head > 0 || a.tail > 0) && (a.vec_n % kE) == t;
    if(!loops && !edges)
        return;
    const uint32_t e = (t + a.start) & (kE - 1);
    E              eng;
#pragma unroll
    for(int k = 0; k < E::kWords; k++)
        eng.w[k] = a.arena[static_cast<size_t>(k) * kE + e];

    using T = typename F::T;
    constexpr unsigned VB = F::ow * sizeof(T);
    uint32_t           in[F::iw];
    T                  out[F::ow];
    unsigned long long j = t;
    // unrolled so that the state words rotate back into place (no register moves per step)
#pragma unroll(E::kUnroll)
    for(; j < a.vec_n; j += kE)
    {
#pragma unroll
        for(unsigned i = 0; i < F::iw; i++)
            in[i] = eng.next();
        g(in, out);
        store_small(a.vec + j * VB, out);
    }
    if(F::ow > 1 && j == a.vec_n)
    {
        T* data = reinterpret_cast<T*>(a.data);
        if(a.head > 0)
        {
            for(unsigned i = 0; i < F::iw; i++)
                in[i] = eng.next();
            g(in, out);
            for(unsigned o = 0; o < a.head; o++)
                data[o] = out[o];
        }
        if(a.tail > 0)
        {
            for(unsigned i = 0; i < F::iw; i++)
                in[i] = eng.next();
            g(in, out);
            for(unsigned o = 0; o < a.tail; o++)
                data[a.n - a.tail + o] = out[o];
        }
    }
#pragma unroll
    for(int k = 0; k < E::kWords; k++)
        a.arena[static_cast<size_t>(k) * kE + e] = eng.w[k];
}

// The same output contract on the host (host generators without a GPU).  Slots are
// independent (distinct engines, distinct output vectors, the head and tail written by one
// slot), so chunks of consecutive slots spread over the host's cores; a chunk keeps its
// engines in a local array and runs round by round (vector j = round * E + slot), so each
// round writes one contiguous run of the output instead of one value every E vectors.
template<class E, class F>
static void stateful_edges_host(const FillArgs& a, const F& f, E& eng)
{
    using T = typename F::T;
    T        out[F::ow];
    uint32_t in[F::iw];
    T*       data = reinterpret_cast<T*>(a.data);
    if(a.head > 0)
    {
        for(unsigned i = 0; i < F::iw; i++)
            in[i] = eng.next();
        f(in, out);
        for(unsigned o = 0; o < a.head; o++)
            data[o] = out[o];
    }
    if(a.tail > 0)
    {
        for(unsigned i = 0; i < F::iw; i++)
            in[i] = eng.next();
        f(in, out);
        for(unsigned o = 0; o < a.tail; o++)
            data[a.n - a.tail + o] = out[o];
    }
}

template<class E>
static void load_engine_host(const FillArgs& a, uint32_t t, E& eng)
{
    const uint32_t e = (t + a.start) & (kE - 1);
    for(int k = 0; k < E::kWords; k++)
        eng.w[k] = a.arena[static_cast<size_t>(k) * kE + e];
}

template<class E>
static void store_engine_host(const FillArgs& a, uint32_t t, const E& eng)
{
    const uint32_t e = (t + a.start) & (kE - 1);
    for(int k = 0; k < E::kWords; k++)
        a.arena[static_cast<size_t>(k) * kE + e] = eng.w[k];
}

template<class E, class F>
static void stateful_fill_host(const FillArgs& a, const F& f)
{
    using T                  = typename F::T;
    constexpr unsigned VB    = F::ow * sizeof(T);
    constexpr uint32_t kRun  = 1024; // slots per chunk
    const bool         edges = F::ow > 1 && (a.head > 0 || a.tail > 0);
    const uint32_t     te    = static_cast<uint32_t>(a.vec_n % kE); // the slot that writes them
    // slots below min(vec_n, E) loop; the edge slot is among them unless vec_n < E
    const unsigned long long active = std::min<unsigned long long>(a.vec_n, kE);
    const unsigned long long chunks = (active + kRun - 1) / kRun;
    host_parallel_for(
        chunks,
        [&](unsigned long long c0, unsigned long long c1) {
            std::vector<E> eng(kRun);
            for(unsigned long long c = c0; c < c1; c++)
            {
                const uint32_t t0 = static_cast<uint32_t>(c * kRun);
                const uint32_t t1 = static_cast<uint32_t>(std::min<unsigned long long>(active, t0 + kRun));
                for(uint32_t t = t0; t < t1; t++)
                    load_engine_host(a, t, eng[t - t0]);
                for(unsigned long long base = 0; base + t0 < a.vec_n; base += kE)
                {
                    const uint32_t last = static_cast<uint32_t>(std::min<unsigned long long>(t1, a.vec_n - base));
                    for(uint32_t t = t0; t < last; t++)
                    {
                        uint32_t in[F::iw];
                        T        out[F::ow];
                        for(unsigned i = 0; i < F::iw; i++)
                            in[i] = eng[t - t0].next();
                        f(in, out);
                        store_small(a.vec + (base + t) * VB, out);
                    }
                }
                if(edges && te >= t0 && te < t1)
                    stateful_edges_host(a, f, eng[te - t0]);
                for(uint32_t t = t0; t < t1; t++)
                    store_engine_host(a, t, eng[t - t0]);
            }
        },
        2);
    if(edges && a.vec_n < kE)
    {
        E eng;
        load_engine_host(a, te, eng);
        stateful_edges_host(a, f, eng);
        store_engine_host(a, te, eng);
    }
}

// ---------------------------------------------------------------------------------------
// Host side: seeding, base states and tables.

using Family = StatefulFamily;

// Device copies of the per-digit jump tables, one upload per (family, device).
struct DeviceTables
{
    std::mutex                 mu;
    std::vector<const void*>   ptr = std::vector<const void*>(64, nullptr);
};

// Host copies of the per-digit jump tables, computed once per family (the source of the
// device uploads and the tables of the CPU path).
struct HostDigitTables
{
    std::vector<uint32_t> t32; // GF(2) families
    std::vector<uint64_t> t64; // MRG families
};

static const HostDigitTables& host_digit_tables(Family fam)
{
    static HostDigitTables t[4];
    static std::once_flag  once[4];
    const int              i = static_cast<int>(fam);
    std::call_once(once[i], [&] {
        HostDigitTables& h = t[i];
        switch(fam)
        {
            case Family::XORWOW: h.t32 = gf2_digit_tables(gf2_pow2(xorwow_step_matrix(), 67)); break;
            case Family::LFSR113: h.t32 = gf2_digit_tables(gf2_pow2(lfsr113_step_matrix(), 55)); break;
            case Family::MRG32K3A:
                h.t64 = mod_digit_tables(mod_pow2(mrg32k3a_step1(), 76), mod_pow2(mrg32k3a_step2(), 76));
                break;
            case Family::MRG31K3P:
                h.t64 = mod_digit_tables(mod_pow2(mrg31k3p_step1(), 72), mod_pow2(mrg31k3p_step2(), 72));
                break;
        }
    });
    return t[i];
}

static const void* digit_tables(Family fam)
{
    static DeviceTables cache[4];
    DeviceTables&       c   = cache[static_cast<int>(fam)];
    const int           dev = device_info().device;
    std::lock_guard<std::mutex> lock(c.mu);
    if(c.ptr[dev])
        return c.ptr[dev];
    const std::vector<uint32_t>& t32 = host_digit_tables(fam).t32;
    const std::vector<uint64_t>& t64 = host_digit_tables(fam).t64;
    void*        d     = nullptr;
    const size_t bytes = t32.empty() ? t64.size() * 8 : t32.size() * 4;
    if(cudaMalloc(&d, bytes) != cudaSuccess)
        return nullptr;
    if(cudaMemcpy(d, t32.empty() ? static_cast<const void*>(t64.data()) : t32.data(), bytes,
                  cudaMemcpyHostToDevice)
       != cudaSuccess)
    {
        cudaFree(d);
        return nullptr;
    }
    c.ptr[dev] = d;
    return d;
}

// XORWOW jump polynomials p_e, e < E (derived at build time by make_xorwow_jump.c and
// embedded by xorwow_data.S), one upload per device.
static const uint32_t* xorwow_jump_polys()
{
    static DeviceTables c;
    const int           dev = device_info().device;
    std::lock_guard<std::mutex> lock(c.mu);
    if(c.ptr[dev])
        return static_cast<const uint32_t*>(c.ptr[dev]);
    const size_t bytes = static_cast<size_t>(rb200_xorwow_jump_end - rb200_xorwow_jump_begin);
    if(bytes != sizeof(uint32_t) * 5 * kE)
        return nullptr;
    void* d = nullptr;
    if(cudaMalloc(&d, bytes) != cudaSuccess)
        return nullptr;
    if(cudaMemcpy(d, rb200_xorwow_jump_begin, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
    {
        cudaFree(d);
        return nullptr;
    }
    c.ptr[dev] = d;
    return static_cast<const uint32_t*>(d);
}

const uint32_t* stateful_xorwow_jump_polys()
{
    return xorwow_jump_polys();
}

void xorwow_word_sequence(const uint32_t* base, uint32_t* seq)
{
    uint32_t x[5];
    std::memcpy(x, base, sizeof(x));
    std::memcpy(seq, x, sizeof(x));
    for(int k = 5; k < kXorwowSeqWords; k++)
    {
        const uint32_t t = x[0] ^ (x[0] >> 2);
        x[0]             = x[1];
        x[1]             = x[2];
        x[2]             = x[3];
        x[3]             = x[4];
        x[4]             = (x[4] ^ (x[4] << 4)) ^ (t ^ (t << 1));
        seq[k]           = x[4];
    }
}

// A^(2^k), k = 0..63, of the one-step map (host offset jumps), computed once per family.
struct PowTables
{
    std::vector<Gf2Matrix> gf2;
    std::vector<ModMatrix> m1, m2;
};

static const PowTables& pow_tables(Family fam)
{
    static PowTables  t[4];
    static std::once_flag once[4];
    const int         i = static_cast<int>(fam);
    std::call_once(once[i], [&] {
        PowTables& p = t[i];
        if(fam == Family::XORWOW || fam == Family::LFSR113)
        {
            Gf2Matrix a = fam == Family::XORWOW ? xorwow_step_matrix() : lfsr113_step_matrix();
            for(int k = 0; k < 64; k++)
            {
                p.gf2.push_back(a);
                a = a.then(a);
            }
        }
        else
        {
            ModMatrix a1 = fam == Family::MRG32K3A ? mrg32k3a_step1() : mrg31k3p_step1();
            ModMatrix a2 = fam == Family::MRG32K3A ? mrg32k3a_step2() : mrg31k3p_step2();
            for(int k = 0; k < 64; k++)
            {
                p.m1.push_back(a1);
                p.m2.push_back(a2);
                a1 = a1.mul(a1);
                a2 = a2.mul(a2);
            }
        }
    });
    return t[i];
}

// Applies A^steps to a state (the engine's discard(steps)); XORWOW also advances its Weyl
// counter d by steps * 362437 (rocrand_xorwow.h:134-145).
static void host_discard(Family fam, uint32_t* s, unsigned long long steps)
{
    const PowTables& p = pow_tables(fam);
    if(fam == Family::XORWOW)
        s[5] += static_cast<uint32_t>(steps) * 362437u;
    for(int k = 0; k < 64 && steps; k++, steps >>= 1)
    {
        if(!(steps & 1))
            continue;
        uint32_t y[6];
        if(fam == Family::XORWOW || fam == Family::LFSR113)
        {
            p.gf2[k].apply(s, y);
            std::memcpy(s, y, sizeof(uint32_t) * p.gf2[k].words);
        }
        else
        {
            p.m1[k].apply(s, y);
            p.m2[k].apply(s + 3, y + 3);
            std::memcpy(s, y, sizeof(uint32_t) * 6);
        }
    }
}

// MRG32k3a seeding arithmetic, wrap-around included (rocrand_mrg32k3a.h:103-120, 262-300).
static uint64_t m32_mod_m1(uint64_t p)
{
    p = 209ull * (p >> 32) + (p & 0xffffffffull);
    return p >= 4294967087ull ? p - 4294967087ull : p;
}
static uint64_t m32_mod_m2(uint64_t p)
{
    p = 22853ull * (p >> 32) + (p & 0xffffffffull);
    p = 22853ull * (p >> 32) + (p & 0xffffffffull);
    return p >= 4294944443ull ? p - 4294944443ull : p;
}
template<uint64_t (*Mod)(uint64_t)>
static uint64_t m32_mod_mul(uint32_t i, uint64_t j, uint64_t m)
{
    long long hi = i / 131072, lo = i - hi * 131072;
    long long t1 = static_cast<long long>(Mod(static_cast<uint64_t>(hi) * j) * 131072);
    long long t2 = static_cast<long long>(Mod(static_cast<uint64_t>(lo) * j));
    lo           = static_cast<long long>(Mod(static_cast<uint64_t>(t1 + t2)));
    if(lo < 0)
        lo += static_cast<long long>(m);
    return static_cast<uint64_t>(lo);
}

// Seeded (engine 0, no jump) state of each family.
static void seeded_state(Family fam, unsigned long long seed, uint4 seed4, uint32_t* s)
{
    switch(fam)
    {
        case Family::XORWOW:
        {
            // rocrand_xorwow.h:100-131
            s[0] = 123456789u;
            s[1] = 362436069u;
            s[2] = 521288629u;
            s[3] = 88675123u;
            s[4] = 5783321u;
            s[5] = 6615241u;
            const uint32_t s0 = static_cast<uint32_t>(seed) ^ 0x2c7f967fu;
            const uint32_t s1 = static_cast<uint32_t>(seed >> 32) ^ 0xa03697cbu;
            const uint32_t t0 = 1228688033u * s0;
            const uint32_t t1 = 2073658381u * s1;
            s[0] += t0;
            s[1] ^= t0;
            s[2] += t1;
            s[3] ^= t1;
            s[4] += t0;
            s[5] += t1 + t0;
            break;
        }
        case Family::MRG32K3A:
        {
            if(seed == 0)
                seed = 12345ull;
            const uint32_t x = static_cast<uint32_t>(seed) ^ 0x55555555u;
            const uint32_t y = static_cast<uint32_t>((seed >> 32) ^ 0xAAAAAAAAull);
            s[0]             = static_cast<uint32_t>(m32_mod_mul<m32_mod_m1>(x, seed, 4294967087ull));
            s[1]             = static_cast<uint32_t>(m32_mod_mul<m32_mod_m1>(y, seed, 4294967087ull));
            s[2]             = static_cast<uint32_t>(m32_mod_mul<m32_mod_m1>(x, seed, 4294967087ull));
            s[3]             = static_cast<uint32_t>(m32_mod_mul<m32_mod_m2>(y, seed, 4294944443ull));
            s[4]             = static_cast<uint32_t>(m32_mod_mul<m32_mod_m2>(x, seed, 4294944443ull));
            s[5]             = static_cast<uint32_t>(m32_mod_mul<m32_mod_m2>(y, seed, 4294944443ull));
            break;
        }
        case Family::MRG31K3P:
        {
            // rocrand_mrg31k3p.h:99-116: (i * j) mod m with the 64-bit product wrapping
            if(seed == 0)
                seed = 12345ull;
            const uint32_t x = static_cast<uint32_t>(seed ^ 0x55555555u);
            const uint32_t y = static_cast<uint32_t>((seed >> 32) ^ 0xAAAAAAAAu);
            s[0]             = static_cast<uint32_t>((x * seed) % 2147483647ull);
            s[1]             = static_cast<uint32_t>((y * seed) % 2147483647ull);
            s[2]             = static_cast<uint32_t>((x * seed) % 2147483647ull);
            s[3]             = static_cast<uint32_t>((y * seed) % 2147462579ull);
            s[4]             = static_cast<uint32_t>((x * seed) % 2147462579ull);
            s[5]             = static_cast<uint32_t>((y * seed) % 2147462579ull);
            break;
        }
        case Family::LFSR113:
            s[0] = seed4.x;
            s[1] = seed4.y;
            s[2] = seed4.z;
            s[3] = seed4.w;
            s[4] = s[5] = 0;
            break;
    }
}

// Base states of engine 0 for engines >= offset % E (base[0]: offset / E steps) and below
// it (base[1]: one step more), xorwow.hpp:45-61 and siblings.
static void bases_of(Family fam, unsigned long long seed, uint4 seed4, unsigned long long offset,
                     uint32_t (&base)[2][6])
{
    unsigned long long jump = offset / kE;
    if(fam == Family::LFSR113)
        jump = static_cast<uint32_t>(jump); // init_lfsr113_engines takes a 32-bit offset
    seeded_state(fam, seed, seed4, base[0]);
    host_discard(fam, base[0], jump);
    std::memcpy(base[1], base[0], sizeof(base[0]));
    if(fam == Family::LFSR113)
    {
        // engines below start skip (uint32)(offset/E) + 1, computed in 32 bits
        seeded_state(fam, seed, seed4, base[1]);
        host_discard(fam, base[1], static_cast<uint32_t>(static_cast<uint32_t>(jump) + 1u));
    }
    else
    {
        host_discard(fam, base[1], 1);
    }
}

// Base states for a position reached by writing `vectors` output vectors of `values` engine
// values each from offset 0: engine e has then stepped values * (vectors / E + (e < vectors %
// E)) times (every vector j is served by engine j mod E), so base[0] skips values * (vectors /
// E) and base[1] (engines below start = vectors % E) values more.
static void bases_at_output(Family fam, unsigned long long seed, uint4 seed4, unsigned long long vectors,
                            unsigned values, uint32_t (&base)[2][6])
{
    const unsigned long long q = vectors / kE;
    seeded_state(fam, seed, seed4, base[0]);
    host_discard(fam, base[0], q * values);
    std::memcpy(base[1], base[0], sizeof(base[0]));
    host_discard(fam, base[1], values);
}

StatefulBases stateful_bases(StatefulFamily fam, unsigned long long seed, unsigned long long offset)
{
    StatefulBases b{};
    uint4         seed4 = make_uint4(2u, 8u, 16u, 128u); // lfsr113.hpp:178-186
    bases_of(fam, seed, seed4, offset, b.base);
    b.start = static_cast<uint32_t>(offset % kE);
    return b;
}

const void* stateful_digit_tables(StatefulFamily fam)
{
    return digit_tables(fam);
}

template<Family kFam>
class StatefulGenerator final : public PseudoGeneratorBase
{
public:
    StatefulGenerator()
    {
        if constexpr(kFam == Family::LFSR113)
            m_seed4 = make_uint4(2u, 8u, 16u, 128u); // lfsr113.hpp:178-186
    }
    ~StatefulGenerator() override
    {
        if(m_arena != nullptr)
            cudaFree(m_arena);
    }

    bool set_host_execution() override { return enable_host(); }

    rocrand_rng_type type() const override
    {
        switch(kFam)
        {
            case Family::XORWOW: return ROCRAND_RNG_PSEUDO_XORWOW;
            case Family::MRG32K3A: return ROCRAND_RNG_PSEUDO_MRG32K3A;
            case Family::MRG31K3P: return ROCRAND_RNG_PSEUDO_MRG31K3P;
            default: return ROCRAND_RNG_PSEUDO_LFSR113;
        }
    }

    rocrand_status set_seed(unsigned long long seed) override
    {
        if constexpr(kFam == Family::LFSR113)
        {
            // lfsr113.hpp:240-255: 16-bit-overlapping words; only x and y get minimums
            uint4 s = make_uint4(static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 16),
                                 static_cast<uint32_t>(seed >> 32), static_cast<uint32_t>(seed >> 48));
            if(s.x < 2u)
                s.x += 2u;
            if(s.y < 8u)
                s.y += 8u;
            m_seed4 = s;
        }
        else if constexpr(kFam == Family::MRG32K3A || kFam == Family::MRG31K3P)
        {
            m_seed = seed == 0 ? 12345ull : seed; // mrg.hpp:236-240
        }
        else
        {
            m_seed = seed;
        }
        m_initialized = false;
        return ROCRAND_STATUS_SUCCESS;
    }

    rocrand_status set_seed_uint4(uint4 seed) override
    {
        if constexpr(kFam == Family::LFSR113)
        {
            // lfsr113.hpp:257-269
            if(seed.x < 2u)
                seed.x += 2u;
            if(seed.y < 8u)
                seed.y += 8u;
            if(seed.z < 16u)
                seed.z += 16u;
            if(seed.w < 128u)
                seed.w += 128u;
            m_seed4       = seed;
            m_initialized = false;
            return ROCRAND_STATUS_SUCCESS;
        }
        else
        {
            (void)seed;
            return ROCRAND_STATUS_TYPE_ERROR;
        }
    }

    rocrand_status set_order(rocrand_ordering order) override
    {
        switch(order)
        {
            case ROCRAND_ORDERING_PSEUDO_SEEDED:
                if(kFam != Family::XORWOW)
                    return ROCRAND_STATUS_OUT_OF_RANGE; // only xorwow.hpp:254-258 lists it
                [[fallthrough]];
            case ROCRAND_ORDERING_PSEUDO_DEFAULT:
            case ROCRAND_ORDERING_PSEUDO_DYNAMIC:
            case ROCRAND_ORDERING_PSEUDO_BEST:
            case ROCRAND_ORDERING_PSEUDO_LEGACY:
                m_order       = order;
                m_initialized = false;
                return ROCRAND_STATUS_SUCCESS;
            default: return ROCRAND_STATUS_OUT_OF_RANGE;
        }
    }

    rocrand_status init() override
    {
        if(m_initialized)
            return ROCRAND_STATUS_SUCCESS;
        // the Poisson tables are allocated here, as the reference's generators do in init(), so
        // that a generate call recorded by a stream capture allocates nothing
        if(m_poisson.reserve() != ROCRAND_STATUS_SUCCESS)
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        if(m_arena == nullptr && !m_host_exec)
        {
            if(cudaMalloc(&m_arena, sizeof(uint32_t) * 6 * kE) != cudaSuccess)
            {
                m_arena = nullptr;
                return ROCRAND_STATUS_ALLOCATION_FAILED;
            }
        }
        InitArgs a{};
        if(m_has_pos)
        {
            m_start = static_cast<uint32_t>(m_pos_vectors % kE);
            bases_at_output(kFam, m_seed, m_seed4, m_pos_vectors, m_pos_values, a.base);
        }
        else
        {
            m_start = static_cast<uint32_t>(m_offset % kE);
            bases_of(kFam, m_seed, m_seed4, m_offset, a.base);
        }
        a.start = m_start;
        a.arena = m_arena;
        if(m_host_exec)
        {
            const rocrand_status hs = init_host(a);
            if(hs == ROCRAND_STATUS_SUCCESS)
                m_initialized = true;
            return hs;
        }
        const unsigned blocks = kE / kBlock;
        if constexpr(kFam == Family::XORWOW)
        {
            const uint32_t* polys = xorwow_jump_polys();
            if(polys == nullptr)
                return ROCRAND_STATUS_ALLOCATION_FAILED;
            XorwowInitArgs x{};
            x.a = a;
            xorwow_word_sequence(a.base[0], x.seq[0]);
            xorwow_word_sequence(a.base[1], x.seq[1]);
            init_xorwow<<<kE / (kBlock * kXorwowInitPerThread), kBlock, 0, m_stream>>>(x, polys);
        }
        else
        {
            const void* tables = digit_tables(kFam);
            if(tables == nullptr)
                return ROCRAND_STATUS_ALLOCATION_FAILED;
            if constexpr(kFam == Family::LFSR113)
                init_gf2<4, 4><<<blocks, kBlock, 0, m_stream>>>(a, static_cast<const uint32_t*>(tables));
            else if constexpr(kFam == Family::MRG32K3A)
                init_mrg<<<blocks, kBlock, 0, m_stream>>>(a, static_cast<const uint64_t*>(tables),
                                                         4294967087ull, 4294944443ull);
            else
                init_mrg<<<blocks, kBlock, 0, m_stream>>>(a, static_cast<const uint64_t*>(tables),
                                                         2147483647ull, 2147462579ull);
        }
        const rocrand_status st = launch_status();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        m_initialized = true;
        return ROCRAND_STATUS_SUCCESS;
    }

    rocrand_status set_offset(unsigned long long offset) override
    {
        m_has_pos = false;
        return PseudoGeneratorBase::set_offset(offset);
    }

    // Output `index` of distribution d: vector V = index / ow was served by engine V mod E,
    // so every engine has stepped iw * (V / E + (e < V % E)) values and the rotation starts at
    // V mod E (xorwow.hpp:385-389 advances start by one per vector).
    rocrand_status set_output_position(Dist d, unsigned long long index) override
    {
        if(d == Dist::U64)
            return ROCRAND_STATUS_TYPE_ERROR;
        DistParams     p;
        unsigned       iw = 0, ow = 1;
        auto           body = [&](auto f) -> rocrand_status {
            iw = decltype(f)::iw;
            ow = decltype(f)::ow;
            return ROCRAND_STATUS_SUCCESS;
        };
        rocrand_status st;
        if constexpr(kFam == Family::MRG32K3A)
            st = with_functor_mrg<Mrg32k3aNorm>(d, p, body);
        else if constexpr(kFam == Family::MRG31K3P)
            st = with_functor_mrg<Mrg31k3pNorm>(d, p, body);
        else
            st = with_functor(d, p, body);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        if(index % ow != 0)
            return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
        m_offset      = 0;
        m_has_pos     = true;
        m_pos_vectors = index / ow;
        m_pos_values  = iw;
        m_initialized = false;
        return ROCRAND_STATUS_SUCCESS;
    }

    rocrand_status generate(void* data, size_t n, Dist d, const DistParams& p) override
    {
        if(d == Dist::U64)
            return ROCRAND_STATUS_TYPE_ERROR;
        rocrand_status st = init();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        if(data == nullptr)
            return ROCRAND_STATUS_SUCCESS;
        const size_t tsize = dist_elem_size(d);
        if(reinterpret_cast<uintptr_t>(data) % tsize != 0)
            return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
        auto body = [&](auto f) -> rocrand_status { return run(f, data, n, tsize); };
        if constexpr(kFam == Family::MRG32K3A)
            return with_functor_mrg<Mrg32k3aNorm>(d, p, body);
        else if constexpr(kFam == Family::MRG31K3P)
            return with_functor_mrg<Mrg31k3pNorm>(d, p, body);
        else
            return with_functor(d, p, body);
    }

    rocrand_status generate_poisson(unsigned int* data, size_t n, double lambda) override
    {
        rocrand_status st = init();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        DistParams p;
        st = m_poisson.get(lambda, m_stream, false, p);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        return generate(data, n, Dist::POISSON, p);
    }

    rocrand_status batch_descriptor(uint32_t dist, double p0, double p1, void* data, size_t n,
                                    BatchReq& r, cudaStream_t stream) override
    {
        if constexpr(kFam != Family::XORWOW && kFam != Family::MRG32K3A)
        {
            return ROCRAND_STATUS_TYPE_ERROR;
        }
        else
        {
            if(m_host_exec)
                return ROCRAND_STATUS_TYPE_ERROR; // the batched fill is a device launch
            rocrand_status st = init();
            if(st != ROCRAND_STATUS_SUCCESS)
                return st;
            r       = BatchReq{};
            r.kind  = kFam == Family::XORWOW ? BK_XORWOW : BK_MRG32K3A;
            r.arena = m_arena;
            r.start = m_start;
            st      = batch_set_dist(r, dist, p0, p1, stream);
            if(st == ROCRAND_STATUS_SUCCESS)
                st = batch_layout(r, data, n);
            if(st != ROCRAND_STATUS_SUCCESS)
                return st;
            unsigned iw, ow;
            batch_widths(r.kind, dist, iw, ow);
            m_start = static_cast<uint32_t>((m_start + (n + ow - 1) / ow) % kE);
            return ROCRAND_STATUS_SUCCESS;
        }
    }

private:
    template<class F>
    rocrand_status run(const F& f, void* data, size_t n, size_t tsize)
    {
        constexpr unsigned ow   = F::ow;
        const uintptr_t    addr = reinterpret_cast<uintptr_t>(data);
        const size_t       mis  = (ow - addr / tsize % ow) % ow;
        FillArgs           a;
        a.arena = m_arena;
        a.start = m_start;
        a.head  = static_cast<uint32_t>(n < mis ? n : mis);
        a.tail  = static_cast<uint32_t>((n - a.head) % ow);
        a.vec_n = (n - a.head) / ow;
        a.n     = n;
        a.data  = static_cast<unsigned char*>(data);
        a.vec   = a.data + mis * tsize;
        using Eng = std::conditional_t<
            kFam == Family::XORWOW, XorwowEngine,
            std::conditional_t<kFam == Family::LFSR113, Lfsr113Engine,
                               std::conditional_t<kFam == Family::MRG32K3A, Mrg32k3aEngine, Mrg31k3pEngine>>>;
        if(n > 0 && m_host_exec)
        {
            a.arena = m_harena.data();
            stateful_fill_host<Eng>(a, f);
        }
        else if(n > 0)
        {
            const size_t smem = table_smem_bytes(f);
            stateful_fill<Eng, F><<<kE / kBlock, kBlock, smem, m_stream>>>(a, f);
            const rocrand_status st = launch_status();
            if(st != ROCRAND_STATUS_SUCCESS)
                return st;
        }
        m_start = static_cast<uint32_t>((m_start + (n + ow - 1) / ow) % kE);
        return ROCRAND_STATUS_SUCCESS;
    }

    // Host execution: engine e = J^e base[e < start] on the host's cores, from the same
    // tables as the device init (the per-digit matrices; XORWOW's jump polynomials).
    rocrand_status init_host(const InitArgs& a)
    {
        m_harena.assign(static_cast<size_t>(6) * kE, 0u);
        uint32_t* arena = m_harena.data();
        if constexpr(kFam == Family::XORWOW)
        {
            const size_t bytes = static_cast<size_t>(rb200_xorwow_jump_end - rb200_xorwow_jump_begin);
            if(bytes != sizeof(uint32_t) * 5 * kE)
                return ROCRAND_STATUS_INTERNAL_ERROR;
            const uint32_t* polys  = reinterpret_cast<const uint32_t*>(rb200_xorwow_jump_begin);
            auto            tables = std::make_unique<XorwowJumpTable[]>(2);
            for(int b = 0; b < 2; b++)
            {
                uint32_t seq[kXorwowSeqWords];
                xorwow_word_sequence(a.base[b], seq);
                xorwow_build_jump_table(tables[b], seq, 0, 1);
            }
            host_parallel_for(kE, [&](unsigned long long e0, unsigned long long e1) {
                for(unsigned long long e = e0; e < e1; e++)
                {
                    const int which = e < a.start ? 1 : 0;
                    uint32_t  x[5];
                    xorwow_jump(tables[which], polys, static_cast<uint32_t>(e), x);
                    for(int w = 0; w < 5; w++)
                        arena[static_cast<size_t>(w) * kE + e] = x[w];
                    arena[static_cast<size_t>(5) * kE + e] = a.base[which][5];
                }
            });
        }
        else
        {
            const HostDigitTables& t = host_digit_tables(kFam);
            host_parallel_for(kE, [&](unsigned long long e0, unsigned long long e1) {
                for(unsigned long long e = e0; e < e1; e++)
                {
                    const int which = e < a.start ? 1 : 0;
                    uint32_t  x[6];
                    std::memcpy(x, a.base[which], sizeof(x));
                    if constexpr(kFam == Family::LFSR113)
                        gf2_jump_digits<4>(t.t32.data(), static_cast<uint32_t>(e), x);
                    else if constexpr(kFam == Family::MRG32K3A)
                        mod_jump_digits(t.t64.data(), 4294967087ull, 4294944443ull, static_cast<uint32_t>(e), x);
                    else
                        mod_jump_digits(t.t64.data(), 2147483647ull, 2147462579ull, static_cast<uint32_t>(e), x);
                    for(int w = 0; w < 6; w++)
                        arena[static_cast<size_t>(w) * kE + e] = x[w];
                }
            });
        }
        return ROCRAND_STATUS_SUCCESS;
    }

    uint4     m_seed4 = {0, 0, 0, 0};
    uint32_t* m_arena = nullptr;
    // engine states of the CPU path (the device arena's layout, in host memory)
    std::vector<uint32_t> m_harena;
    uint32_t  m_start = 0;
    // rocrand_b200_set_output_position: engines placed after m_pos_vectors vectors of
    // m_pos_values values each (replaces the offset until the next set_offset)
    bool               m_has_pos     = false;
    unsigned long long m_pos_vectors = 0;
    unsigned           m_pos_values  = 1;
};

rocrand_generator_base_type* make_stateful(rocrand_rng_type t)
{
    switch(t)
    {
        case ROCRAND_RNG_PSEUDO_DEFAULT:
        case ROCRAND_RNG_PSEUDO_XORWOW: return new StatefulGenerator<Family::XORWOW>();
        case ROCRAND_RNG_PSEUDO_MRG32K3A: return new StatefulGenerator<Family::MRG32K3A>();
        case ROCRAND_RNG_PSEUDO_MRG31K3P: return new StatefulGenerator<Family::MRG31K3P>();
        case ROCRAND_RNG_PSEUDO_LFSR113: return new StatefulGenerator<Family::LFSR113>();
        default: return nullptr;
    }
}

} // namespace rb200
