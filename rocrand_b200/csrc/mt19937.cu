// mt19937.cu -- MT19937: 8192 state-parallel generators, eight lanes each.
//
// Output order (library/src/rng/mt19937.hpp:306-662, mt19937_octo_engine.hpp): 65536 threads
// (256 x 256, config/config_defaults.hpp:76-80), eight per generator.  Lane t of generator g
// owns 78 of the generator's 624 state words ("slots"): slot 0 is word
// {0,113,170,283,340,397,510,567}[t] and slot 1+7i+j is word
// {1,57,114,171,227,284,341,398,454,511,568}[i] + 7t + j.  Input unit u of a call (one
// distribution call of iw words) is slot group (u % full) / 65536 of thread u % 65536 in
// round u / full, full = 65536 * (78 / iw); round 0 is the state the previous call left
// when it stopped mid-round, otherwise a fresh twist.
//
// B200 layout: the arena holds slot j of thread t at arena[j * 65536 + t] (each warp's
// load/store of one slot is one 128-byte line).  A thread keeps its 78 words in registers
// for the whole call and twists them with width-8 warp shuffles in the dependency order of
// the sequential recurrence; the grid is 1024 blocks of 64 threads, so all 65536 lanes are
// resident at once on 148 SMs (7 blocks per SM).
//
// Seeding (mt19937.hpp:83-206): generator e starts from the Knuth state of
// (seed >> 32) ^ seed advanced by e * 2^1000 steps.  A jump polynomial p applied to a state
// whose continuation is x gives word k = XOR of x[i + k] over the set coefficients i of p,
// so each block extends its start state to 20560 words in shared memory and lets 624
// threads accumulate one word each.  The polynomials (x^(i 2^1000) and x^(256 i 2^1000)
// mod the characteristic polynomial) are derived at build time by
// rocrand_b200/data/make_mt19937_jump.c and embedded by mt19937_data.S.
#include "common.hpp"
#include "dist.cuh"
#include "generators.hpp"
#include "host_exec.hpp"
#include "launch.cuh"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

extern "C" const uint32_t rb200_mt19937_jump_begin[];
extern "C" const uint32_t rb200_mt19937_jump_end[];

namespace rb200
{
namespace
{

constexpr unsigned kMtN       = 624;
constexpr unsigned kMtM       = 397;
constexpr unsigned kMtGens    = 8192;
constexpr unsigned kMtThreads = kMtGens * 8; // 65536
constexpr unsigned kMtSlots   = 78;
constexpr unsigned kMtSeq     = 19937 + kMtN - 1; // a state and the 19936 words after it
constexpr unsigned kMtPolys   = 255 + 31;
constexpr unsigned kMtBlock   = 64;
constexpr unsigned kJumpBlock = 640;
constexpr uint32_t kFullMask  = 0xffffffffu;

__host__ __device__ __forceinline__ uint32_t mt_mix(uint32_t a, uint32_t b, uint32_t m)
{
    const uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
    return m ^ (y >> 1) ^ ((0u - (y & 1u)) & 0x9908b0dfu);
}

__host__ __device__ __forceinline__ uint32_t mt_temper(uint32_t y)
{
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

__device__ __forceinline__ uint32_t from_lane(uint32_t v, int src)
{
    return __shfl_sync(kFullMask, v, src, 8);
}

// Twists the seven-word group G (slots 1+7G..7+7G); its m-terms are the same positions of
// group M, and `after` is the word that follows the group (lane 7's successor).
template<int G, int M>
__device__ __forceinline__ void twist_group(uint32_t (&r)[kMtSlots], unsigned lane, uint32_t after)
{
    constexpr int b    = 1 + 7 * G;
    constexpr int m    = 1 + 7 * M;
    uint32_t      next = __shfl_down_sync(kFullMask, r[b], 1, 8);
    next               = lane == 7 ? after : next;
#pragma unroll
    for(int j = 0; j < 6; j++)
        r[b + j] = mt_mix(r[b + j], r[b + j + 1], r[m + j]);
    r[b + 6] = mt_mix(r[b + 6], next, r[m + 6]);
}

// Twists the slot-0 word of lane L.
template<unsigned L>
__device__ __forceinline__ void twist_single(uint32_t (&r)[kMtSlots], unsigned lane, uint32_t next,
                                             uint32_t mterm)
{
    const uint32_t v = mt_mix(r[0], next, mterm);
    r[0]             = lane == L ? v : r[0];
}

// One full twist of the 624 words spread over the eight lanes, in the order of the
// sequential recurrence mt[i] = f(mt[i], mt[i+1], mt[i+397 mod 624]): words 0..226 read old
// m-terms, words 227..623 read the new words 0..396, word 623 reads the new word 0.
__device__ __forceinline__ void mt_twist(uint32_t (&r)[kMtSlots], unsigned lane)
{
    twist_single<0>(r, lane, r[1], from_lane(r[0], 5));                // 0:   next 1, m 397
    twist_group<0, 7>(r, lane, from_lane(r[8], 0));                    // 1..56,   after 57
    twist_group<1, 8>(r, lane, from_lane(r[0], 1));                    // 57..112, after 113
    twist_single<1>(r, lane, from_lane(r[15], 0), from_lane(r[0], 6)); // 113: next 114, m 510
    twist_group<2, 9>(r, lane, from_lane(r[0], 2));                    // 114..169, after 170
    twist_single<2>(r, lane, from_lane(r[22], 0), from_lane(r[0], 7)); // 170: next 171, m 567
    twist_group<3, 10>(r, lane, from_lane(r[29], 0));                  // 171..226, after 227
    {
        // 227..282: m-terms are the new words 7t .. 7t+6 (word 7t is lane t-1's slot 7,
        // or word 0 for lane 0)
        const uint32_t after = from_lane(r[0], 3); // 283
        uint32_t       next  = __shfl_down_sync(kFullMask, r[29], 1, 8);
        next                 = lane == 7 ? after : next;
        uint32_t first       = __shfl_up_sync(kFullMask, r[7], 1, 8);
        first                = lane == 0 ? r[0] : first;
        r[29]                = mt_mix(r[29], r[30], first);
#pragma unroll
        for(int j = 1; j < 6; j++)
            r[29 + j] = mt_mix(r[29 + j], r[30 + j], r[j]);
        r[35] = mt_mix(r[35], next, r[6]);
    }
    twist_single<3>(r, lane, from_lane(r[36], 0), from_lane(r[7], 7)); // 283: next 284, m 56
    twist_group<5, 1>(r, lane, from_lane(r[0], 4));                    // 284..339, after 340
    twist_single<4>(r, lane, from_lane(r[43], 0), from_lane(r[0], 1)); // 340: next 341, m 113
    twist_group<6, 2>(r, lane, from_lane(r[0], 5));                    // 341..396, after 397
    twist_single<5>(r, lane, from_lane(r[50], 0), from_lane(r[0], 2)); // 397: next 398, m 170
    twist_group<7, 3>(r, lane, from_lane(r[57], 0));                   // 398..453, after 454
    twist_group<8, 4>(r, lane, from_lane(r[0], 6));                    // 454..509, after 510
    twist_single<6>(r, lane, from_lane(r[64], 0), from_lane(r[0], 3)); // 510: next 511, m 283
    twist_group<9, 5>(r, lane, from_lane(r[0], 7));                    // 511..566, after 567
    twist_single<7>(r, lane, from_lane(r[71], 0), from_lane(r[0], 4)); // 567: next 568, m 340
    twist_group<10, 6>(r, lane, from_lane(r[0], 0));                   // 568..623, after 0 (new)
}

// Lane and slot of state word k.
__device__ __forceinline__ void word_home(unsigned k, unsigned& lane, unsigned& slot)
{
    constexpr unsigned kSingle[8] = {0, 113, 170, 283, 340, 397, 510, 567};
    constexpr unsigned kGroup[11] = {1, 57, 114, 171, 227, 284, 341, 398, 454, 511, 568};
#pragma unroll
    for(unsigned t = 0; t < 8; t++)
    {
        if(k == kSingle[t])
        {
            lane = t;
            slot = 0;
            return;
        }
    }
    unsigned i = 0;
#pragma unroll
    for(unsigned g = 1; g < 11; g++)
        i = k >= kGroup[g] ? g : i;
    const unsigned d = k - kGroup[i];
    lane             = d / 7;
    slot             = 1 + 7 * i + d % 7;
}

// XOR of x[i + k] over the set coefficients i of `poly` (all threads read the same bits).
__device__ __forceinline__ uint32_t apply_poly(const uint32_t* poly, const uint32_t* x, unsigned k)
{
    uint32_t acc = 0;
    for(unsigned w = 0; w < kMtN; w++)
    {
        uint32_t        bits = poly[w];
        const uint32_t* base = x + 32 * w + k;
        while(bits)
        {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            acc ^= base[b];
        }
    }
    return acc;
}

// Extends the state sh[0..623] to kMtSeq words in place (227 words per step: word k reads
// k-624, k-623 and k-227).
__device__ __forceinline__ void extend_sequence(uint32_t* sh)
{
    for(unsigned c = kMtN; c < kMtSeq; c += kMtN - kMtM)
    {
        const unsigned k = c + threadIdx.x;
        if(threadIdx.x < kMtN - kMtM && k < kMtSeq)
            sh[k] = mt_mix(sh[k - kMtN], sh[k - kMtN + 1], sh[k - (kMtN - kMtM)]);
        __syncthreads();
    }
}

// Block e0 = 1..255: the seed state advanced by e0 * 2^1000 (first radix-256 digit).
__global__ __launch_bounds__(kJumpBlock) void mt_jump_low(const uint32_t* __restrict__ seed_state,
                                                         const uint32_t* __restrict__ polys,
                                                         uint32_t* __restrict__ low_states)
{
    extern __shared__ uint32_t sh[];
    uint32_t*      poly = sh + kMtSeq;
    const unsigned e0   = blockIdx.x + 1;
    for(unsigned k = threadIdx.x; k < kMtN; k += blockDim.x)
    {
        sh[k]   = seed_state[k];
        poly[k] = polys[(e0 - 1) * kMtN + k];
    }
    __syncthreads();
    extend_sequence(sh);
    if(threadIdx.x < kMtN)
        low_states[e0 * kMtN + threadIdx.x] = apply_poly(poly, sh, threadIdx.x);
}

// Block e = 0..8191: generator e's start state (second digit e / 256 applied to the
// first-digit state of e % 256), scattered into the lane/slot arena.
__global__ __launch_bounds__(kJumpBlock) void mt_jump_high(const uint32_t* __restrict__ seed_state,
                                                          const uint32_t* __restrict__ low_states,
                                                          const uint32_t* __restrict__ polys,
                                                          uint32_t* __restrict__ arena)
{
    extern __shared__ uint32_t sh[];
    uint32_t*       poly = sh + kMtSeq;
    const unsigned  e    = blockIdx.x;
    const unsigned  e0 = e % 256, e1 = e / 256;
    const uint32_t* src  = e0 == 0 ? seed_state : low_states + e0 * kMtN;
    for(unsigned k = threadIdx.x; k < kMtN; k += blockDim.x)
    {
        sh[k] = src[k];
        if(e1 != 0)
            poly[k] = polys[(255 + e1 - 1) * kMtN + k];
    }
    __syncthreads();
    uint32_t word = 0;
    if(e1 != 0)
    {
        extend_sequence(sh);
        if(threadIdx.x < kMtN)
            word = apply_poly(poly, sh, threadIdx.x);
    }
    else if(threadIdx.x < kMtN)
    {
        word = sh[threadIdx.x];
    }
    if(threadIdx.x < kMtN)
    {
        unsigned lane, slot;
        word_home(threadIdx.x, lane, slot);
        arena[slot * kMtThreads + e * 8 + lane] = word;
    }
}

struct MtArgs
{
    uint32_t*          arena;
    unsigned char*     data;
    unsigned char*     vec;
    unsigned long long n, vec_n, total; // total = vec_n + (head or tail ? 1 : 0)
    uint32_t           start;           // first unit of the call within the current round
    uint32_t           full;            // units per round
    uint32_t           rounds;          // rounds the call touches
    uint32_t           twist_first;     // round 0 needs a twist (start == 0)
    uint32_t           head, tail;
};

template<class T, unsigned N>
__device__ __forceinline__ void store_vec(unsigned char* p, const T (&v)[N])
{
    constexpr unsigned VB = sizeof(T) * N;
    if constexpr(VB == 4)
    {
        uint32_t w;
        memcpy(&w, v, 4);
        __stcs(reinterpret_cast<unsigned int*>(p), w);
    }
    else if constexpr(VB == 8)
    {
        uint2 w;
        memcpy(&w, v, 8);
        __stcs(reinterpret_cast<uint2*>(p), w);
    }
    else
    {
        static_assert(VB == 16, "vector size");
        uint4 w;
        memcpy(&w, v, 16);
        __stcs(reinterpret_cast<uint4*>(p), w);
    }
}

// One input unit: tempered slots G*iw .. G*iw+iw-1 through the distribution.
template<unsigned G, class F>
__device__ __forceinline__ void unit_values(const F& f, const uint32_t (&r)[kMtSlots],
                                            typename F::T (&out)[F::ow])
{
    uint32_t in[F::iw];
#pragma unroll
    for(unsigned i = 0; i < F::iw; i++)
        in[i] = mt_temper(r[G * F::iw + i]);
    f(in, out);
}

// A thread's input units of a round, from its 78 slots in registers (the short transforms;
// the long ones are staged through shared memory, mt_round_staged).
template<class F>
struct RegUnits
{
    using Fn = F;
    const F&        f;
    const uint32_t (&r)[kMtSlots];
    template<unsigned G>
    __device__ __forceinline__ void get(typename F::T (&out)[F::ow]) const
    {
        unit_values<G>(f, r, out);
    }
};

// Transforms long enough that the state is staged through shared memory for them (the
// normal and log-normal outputs: Box-Muller on every pair).
template<class F>
constexpr bool kMtStaged = std::is_same<F, FnNormalD>::value || std::is_same<F, FnLogNormalD>::value
                           || std::is_same<F, FnNormalF>::value || std::is_same<F, FnLogNormalF>::value
                           || std::is_same<F, FnNormalH>::value || std::is_same<F, FnLogNormalH>::value;

// Units a lane transforms side by side in a staged round inside the call: four fp64
// Box-Muller chains, three fp32 / half ones.
template<class F>
constexpr unsigned kMtUnitsPerStep
    = (std::is_same<F, FnNormalD>::value || std::is_same<F, FnLogNormalD>::value) ? 4u : 3u;

// Shared memory of one block of mt_fill: the distribution's table, or the staged state.
template<class F>
inline size_t mt_fill_smem(const F& f)
{
    return kMtStaged<F> ? sizeof(uint32_t) * kMtSlots * kMtBlock : table_smem_bytes(f);
}

// A round whose units all lie inside the call: every slot group is stored.
template<class U, unsigned... G>
__device__ __forceinline__ void round_interior(const U& u, const MtArgs& a, long long q0,
                                               std::integer_sequence<unsigned, G...>)
{
    using T               = typename U::Fn::T;
    constexpr unsigned ow = U::Fn::ow;
    constexpr unsigned VB = sizeof(T) * ow;
    (
        [&] {
            T out[ow];
            u.template get<G>(out);
            store_vec(a.vec + static_cast<unsigned long long>(q0 + G * kMtThreads) * VB, out);
        }(),
        ...);
}

// The first or last round of a call: units outside the call are skipped, and the one
// extra unit writes the head and tail.
template<class U, unsigned... G>
__device__ __forceinline__ void round_edge(const U& u, const MtArgs& a, long long q0,
                                           std::integer_sequence<unsigned, G...>)
{
    using T               = typename U::Fn::T;
    constexpr unsigned ow = U::Fn::ow;
    constexpr unsigned VB = sizeof(T) * ow;
    (
        [&] {
            const long long q = q0 + static_cast<long long>(G) * kMtThreads;
            if(q < 0 || static_cast<unsigned long long>(q) >= a.total)
                return;
            T out[ow];
            u.template get<G>(out);
            if(static_cast<unsigned long long>(q) < a.vec_n)
            {
                store_vec(a.vec + static_cast<unsigned long long>(q) * VB, out);
                return;
            }
            // the extra unit: head from its front, tail from its back, the tail written
            // downwards from the end (mt19937.hpp:404-430)
            T* data = reinterpret_cast<T*>(a.data);
#pragma unroll
            for(unsigned o = 0; o < ow; o++)
            {
                if(o < a.head)
                    data[o] = out[o];
                if(static_cast<int>(o) > static_cast<int>(ow) - static_cast<int>(a.tail) - 1)
                    data[a.n + (ow - a.tail - 1) - o] = out[o];
            }
        }(),
        ...);
}

// One input unit of a staged round: tempered slots G*iw .. G*iw+iw-1 through F.
template<class F>
__device__ __forceinline__ void staged_unit(const F& f, const uint32_t* s, unsigned G,
                                            typename F::T (&out)[F::ow])
{
    uint32_t in[F::iw];
#pragma unroll
    for(unsigned i = 0; i < F::iw; i++)
        in[i] = mt_temper(s[(G * F::iw + i) * kMtBlock]);
    f(in, out);
}

// A round whose slots were staged in shared memory (slot j of this thread at s[j * 64]):
// the slot groups are a loop, not an unrolled sequence, so the transform's code stays in the
// instruction cache.  A round inside the call takes kMtUnitsPerStep units per iteration with
// no branch between them, so their transform chains interleave (14 warps per SM hold every
// MT lane: the latency is hidden by the lane's own independent work); the call's first and
// last rounds take one unit at a time and skip the units outside the call.
template<class F>
__device__ __forceinline__ void mt_round_staged(const F& f, const uint32_t* s, const MtArgs& a, uint32_t rho)
{
    using T                = typename F::T;
    constexpr unsigned per = kMtSlots / F::iw;
    constexpr unsigned ow  = F::ow;
    constexpr unsigned VB  = sizeof(T) * ow;
    const unsigned     tid = blockIdx.x * kMtBlock + threadIdx.x;
    const long long    base = static_cast<long long>(rho) * a.full - a.start;
    const long long    q0   = base + tid;
    if(base >= 0 && static_cast<unsigned long long>(base) + a.full <= a.total)
    {
        constexpr unsigned U = kMtUnitsPerStep<F>;
        unsigned           G = 0;
#pragma unroll 1
        for(; G + U <= per; G += U)
        {
            T o[U][ow];
#pragma unroll
            for(unsigned u = 0; u < U; u++)
                staged_unit(f, s, G + u, o[u]);
#pragma unroll
            for(unsigned u = 0; u < U; u++)
                store_vec(a.vec + static_cast<unsigned long long>(q0 + (G + u) * kMtThreads) * VB, o[u]);
        }
#pragma unroll 1
        for(; G < per; G++)
        {
            T o0[ow];
            staged_unit(f, s, G, o0);
            store_vec(a.vec + static_cast<unsigned long long>(q0 + G * kMtThreads) * VB, o0);
        }
        return;
    }
#pragma unroll 1
    for(unsigned G = 0; G < per; G++)
    {
        const long long q = q0 + static_cast<long long>(G) * kMtThreads;
        if(q < 0 || static_cast<unsigned long long>(q) >= a.total)
            continue;
        T out[ow];
        staged_unit(f, s, G, out);
        if(static_cast<unsigned long long>(q) < a.vec_n)
        {
            store_vec(a.vec + static_cast<unsigned long long>(q) * VB, out);
            continue;
        }
        // the extra unit: head from its front, tail from its back, the tail written
        // downwards from the end (mt19937.hpp:404-430)
        T* data = reinterpret_cast<T*>(a.data);
#pragma unroll
        for(unsigned o = 0; o < ow; o++)
        {
            if(o < a.head)
                data[o] = out[o];
            if(static_cast<int>(o) > static_cast<int>(ow) - static_cast<int>(a.tail) - 1)
                data[a.n + (ow - a.tail - 1) - o] = out[o];
        }
    }
}

template<class U>
__device__ __forceinline__ void mt_round(const U& u, const MtArgs& a, uint32_t rho)
{
    constexpr unsigned per = kMtSlots / U::Fn::iw;
    using Groups           = std::make_integer_sequence<unsigned, per>;
    const unsigned tid     = blockIdx.x * kMtBlock + threadIdx.x;
    // q of slot group 0 for thread 0 of this round (negative before the call's start)
    const long long base = static_cast<long long>(rho) * a.full - a.start;
    const long long q0   = base + tid;
    if(base >= 0 && static_cast<unsigned long long>(base) + a.full <= a.total)
        round_interior(u, a, q0, Groups{});
    else
        round_edge(u, a, q0, Groups{});
}

template<class F>
__global__ __launch_bounds__(kMtBlock, 7) void mt_fill(MtArgs a, F fw)
{
    extern __shared__ unsigned char smem[];
    const F        f    = stage_table(fw, smem);
    const unsigned tid  = blockIdx.x * kMtBlock + threadIdx.x;
    const unsigned lane = threadIdx.x & 7u;

    uint32_t r[kMtSlots];
#pragma unroll
    for(unsigned j = 0; j < kMtSlots; j++)
        r[j] = a.arena[j * kMtThreads + tid];

    for(uint32_t rho = 0; rho < a.rounds; rho++)
    {
        if(rho > 0 || a.twist_first)
            mt_twist(r, lane);
        if constexpr(kMtStaged<F>)
        {
            // the thread's own slots, one bank each (slot j of thread t at word j * 64 + t)
            uint32_t* s = reinterpret_cast<uint32_t*>(smem) + threadIdx.x;
#pragma unroll
            for(unsigned j = 0; j < kMtSlots; j++)
                s[j * kMtBlock] = r[j];
            // the registers are dead from here: the compiler must read the slots back
            asm volatile("" ::: "memory");
            mt_round_staged(f, s, a, rho);
            asm volatile("" ::: "memory");
#pragma unroll
            for(unsigned j = 0; j < kMtSlots; j++)
                r[j] = s[j * kMtBlock];
        }
        else
        {
            mt_round(RegUnits<F>{f, r}, a, rho);
        }
    }
    if(a.rounds > 1 || (a.rounds == 1 && a.twist_first))
    {
#pragma unroll
        for(unsigned j = 0; j < kMtSlots; j++)
            a.arena[j * kMtThreads + tid] = r[j];
    }
}

// Jump polynomials on each device, uploaded once.
const uint32_t* device_jump_polys()
{
    static std::mutex                   mu;
    static std::vector<const uint32_t*> ptr(64, nullptr);
    const int                           dev = device_info().device;
    std::lock_guard<std::mutex>         lock(mu);
    if(ptr[dev])
        return ptr[dev];
    const size_t words = static_cast<size_t>(rb200_mt19937_jump_end - rb200_mt19937_jump_begin);
    if(words != static_cast<size_t>(kMtPolys) * kMtN)
        return nullptr;
    void* d = nullptr;
    if(cudaMalloc(&d, words * sizeof(uint32_t)) != cudaSuccess)
        return nullptr;
    if(cudaMemcpy(d, rb200_mt19937_jump_begin, words * sizeof(uint32_t), cudaMemcpyHostToDevice)
       != cudaSuccess)
    {
        cudaFree(d);
        return nullptr;
    }
    ptr[dev] = static_cast<const uint32_t*>(d);
    return ptr[dev];
}

// ---- CPU path of the host generators: the same output order on the host's cores ----

// State word held by slot `slot` of lane `lane` (the inverse of word_home).
inline unsigned slot_word(unsigned lane, unsigned slot)
{
    constexpr unsigned kSingle[8] = {0, 113, 170, 283, 340, 397, 510, 567};
    constexpr unsigned kGroup[11] = {1, 57, 114, 171, 227, 284, 341, 398, 454, 511, 568};
    if(slot == 0)
        return kSingle[lane];
    return kGroup[(slot - 1) / 7] + 7 * lane + (slot - 1) % 7;
}

// The sequential recurrence in place: word i reads word i + 1 and word i + 397 (mod 624),
// the later ones already new -- the order mt_twist follows across its lanes.
inline void mt_twist_host(uint32_t* s)
{
    for(unsigned i = 0; i < kMtN; i++)
        s[i] = mt_mix(s[i], s[(i + 1) % kMtN], s[(i + kMtM) % kMtN]);
}

// x[0..623] extended to kMtSeq words (the host form of extend_sequence).
inline void mt_sequence_host(const uint32_t* state, uint32_t* x)
{
    std::memcpy(x, state, sizeof(uint32_t) * kMtN);
    for(unsigned k = kMtN; k < kMtSeq; k++)
        x[k] = mt_mix(x[k - kMtN], x[k - kMtN + 1], x[k - (kMtN - kMtM)]);
}

// out[k] = XOR of x[i + k] over the set coefficients i of `poly` (apply_poly for all 624
// words at once: one pass over the sequence per coefficient).
inline void mt_apply_poly_host(const uint32_t* poly, const uint32_t* x, uint32_t* out)
{
    std::memset(out, 0, sizeof(uint32_t) * kMtN);
    for(unsigned w = 0; w < kMtN; w++)
    {
        for(uint32_t bits = poly[w]; bits; bits &= bits - 1)
        {
            const uint32_t* src = x + 32 * w + static_cast<unsigned>(__builtin_ctz(bits));
            for(unsigned k = 0; k < kMtN; k++)
                out[k] ^= src[k];
        }
    }
}

// Start states of the 8192 generators, word k of generator e at states[e * 624 + k]: the
// same two radix-256 jump digits as mt_jump_low and mt_jump_high.
inline void mt_init_host(const uint32_t* seed_state, uint32_t* states)
{
    const uint32_t*       polys = rb200_mt19937_jump_begin;
    std::vector<uint32_t> x0(kMtSeq);
    mt_sequence_host(seed_state, x0.data());
    std::vector<uint32_t> low(static_cast<size_t>(256) * kMtN);
    std::memcpy(low.data(), seed_state, sizeof(uint32_t) * kMtN);
    host_parallel_for(
        255,
        [&](unsigned long long b, unsigned long long e) {
            for(unsigned long long e0 = b + 1; e0 <= e; e0++)
                mt_apply_poly_host(polys + (e0 - 1) * kMtN, x0.data(), low.data() + e0 * kMtN);
        },
        2);
    host_parallel_for(
        kMtGens,
        [&](unsigned long long b, unsigned long long e) {
            std::vector<uint32_t> y(kMtSeq);
            for(unsigned long long g = b; g < e; g++)
            {
                const uint32_t* src = low.data() + (g % 256) * kMtN;
                const unsigned  e1  = static_cast<unsigned>(g / 256);
                if(e1 == 0)
                {
                    std::memcpy(states + g * kMtN, src, sizeof(uint32_t) * kMtN);
                    continue;
                }
                mt_sequence_host(src, y.data());
                mt_apply_poly_host(polys + static_cast<size_t>(255 + e1 - 1) * kMtN, y.data(),
                                   states + g * kMtN);
            }
        },
        2);
}

// mt_fill on the host: chunks of consecutive generators run round by round with mt_fill's
// unit numbering, skipping and extra unit; within a round, slot group G of the chunk's lanes
// is one contiguous run of units (unit = round base + lane index + G * 65536), written in
// order.  Chunks are independent.
template<class F>
void mt_fill_host(const MtArgs& a, const F& f, uint32_t* states)
{
    using T                    = typename F::T;
    constexpr unsigned iw      = F::iw;
    constexpr unsigned ow      = F::ow;
    constexpr unsigned per     = kMtSlots / iw;
    constexpr unsigned VB      = sizeof(T) * ow;
    constexpr unsigned kGenRun = 64; // generators per chunk (512 lanes)
    host_parallel_for(
        kMtGens / kGenRun,
        [&](unsigned long long c0, unsigned long long c1) {
            for(unsigned long long c = c0; c < c1; c++)
            {
                const unsigned long long g0 = c * kGenRun;
                for(uint32_t rho = 0; rho < a.rounds; rho++)
                {
                    if(rho > 0 || a.twist_first)
                        for(unsigned long long g = g0; g < g0 + kGenRun; g++)
                            mt_twist_host(states + g * kMtN);
                    const long long base = static_cast<long long>(rho) * a.full - a.start;
                    for(unsigned G = 0; G < per; G++)
                    {
                        for(unsigned long long g = g0; g < g0 + kGenRun; g++)
                        {
                            const uint32_t* s = states + g * kMtN;
                            for(unsigned lane = 0; lane < 8; lane++)
                            {
                                const long long q = base + static_cast<long long>(g * 8 + lane)
                                                    + static_cast<long long>(G) * kMtThreads;
                                if(q < 0 || static_cast<unsigned long long>(q) >= a.total)
                                    continue;
                                uint32_t in[iw];
                                for(unsigned i = 0; i < iw; i++)
                                    in[i] = mt_temper(s[slot_word(lane, G * iw + i)]);
                                T out[ow];
                                f(in, out);
                                if(static_cast<unsigned long long>(q) < a.vec_n)
                                {
                                    std::memcpy(a.vec + static_cast<unsigned long long>(q) * VB, out, VB);
                                    continue;
                                }
                                T* data = reinterpret_cast<T*>(a.data);
                                for(unsigned o = 0; o < ow; o++)
                                {
                                    if(o < a.head)
                                        data[o] = out[o];
                                    if(static_cast<int>(o) > static_cast<int>(ow) - static_cast<int>(a.tail) - 1)
                                        data[a.n + (ow - a.tail - 1) - o] = out[o];
                                }
                            }
                        }
                    }
                }
            }
        },
        2);
}

class Mt19937Generator final : public PseudoGeneratorBase
{
public:
    ~Mt19937Generator() override
    {
        if(m_arena != nullptr)
            cudaFree(m_arena);
    }

    bool set_host_execution() override { return enable_host(); }

    rocrand_rng_type type() const override { return ROCRAND_RNG_PSEUDO_MT19937; }

    // mt19937.hpp:758-763: MT19937 has no offset
    rocrand_status set_offset(unsigned long long offset) override
    {
        (void)offset;
        return ROCRAND_STATUS_TYPE_ERROR;
    }

    // mt19937.hpp:765-780
    rocrand_status set_order(rocrand_ordering order) override
    {
        switch(order)
        {
            case ROCRAND_ORDERING_PSEUDO_DEFAULT:
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
        if(m_host_exec)
        {
            if(static_cast<size_t>(rb200_mt19937_jump_end - rb200_mt19937_jump_begin)
               != static_cast<size_t>(kMtPolys) * kMtN)
                return ROCRAND_STATUS_INTERNAL_ERROR;
            uint32_t s[kMtN];
            s[0] = static_cast<uint32_t>((m_seed >> 32) ^ m_seed);
            for(uint32_t i = 1; i < kMtN; i++)
                s[i] = 1812433253u * (s[i - 1] ^ (s[i - 1] >> 30)) + i;
            m_hstate.assign(static_cast<size_t>(kMtGens) * kMtN, 0u);
            mt_init_host(s, m_hstate.data());
            m_start       = 0;
            m_prev_iw     = 0;
            m_initialized = true;
            return ROCRAND_STATUS_SUCCESS;
        }
        const uint32_t* polys = device_jump_polys();
        if(polys == nullptr)
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        constexpr size_t kArenaWords = static_cast<size_t>(kMtSlots) * kMtThreads;
        constexpr size_t kLowWords   = 256 * kMtN;
        if(m_arena == nullptr)
        {
            if(cudaMalloc(&m_arena, sizeof(uint32_t) * (kArenaWords + kLowWords + kMtN))
               != cudaSuccess)
            {
                m_arena = nullptr;
                return ROCRAND_STATUS_ALLOCATION_FAILED;
            }
        }
        uint32_t* low  = m_arena + kArenaWords;
        uint32_t* seed = low + kLowWords;
        // Knuth initialisation of (seed >> 32) ^ seed (mt19937.hpp:107-116)
        uint32_t s[kMtN];
        s[0] = static_cast<uint32_t>((m_seed >> 32) ^ m_seed);
        for(uint32_t i = 1; i < kMtN; i++)
            s[i] = 1812433253u * (s[i - 1] ^ (s[i - 1] >> 30)) + i;
        // pageable source: the copy has read it when cudaMemcpyAsync returns
        if(cudaMemcpyAsync(seed, s, sizeof(s), cudaMemcpyHostToDevice, m_stream) != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        const size_t smem = sizeof(uint32_t) * (kMtSeq + kMtN);
        if(cudaFuncSetAttribute(mt_jump_low, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem))
               != cudaSuccess
           || cudaFuncSetAttribute(mt_jump_high, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem))
                  != cudaSuccess)
            return ROCRAND_STATUS_LAUNCH_FAILURE;
        mt_jump_low<<<255, kJumpBlock, smem, m_stream>>>(seed, polys, low);
        rocrand_status st = launch_status();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        mt_jump_high<<<kMtGens, kJumpBlock, smem, m_stream>>>(seed, low, polys, m_arena);
        st = launch_status();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        m_start       = 0;
        m_prev_iw     = 0;
        m_initialized = true;
        return ROCRAND_STATUS_SUCCESS;
    }

    rocrand_status generate(void* data, size_t n, Dist d, const DistParams& p) override
    {
        if(d == Dist::U64)
            return ROCRAND_STATUS_TYPE_ERROR; // mt19937.hpp:1044-1060
        rocrand_status st = init();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        if(data == nullptr)
            return ROCRAND_STATUS_SUCCESS;
        const size_t tsize = dist_elem_size(d);
        if(reinterpret_cast<uintptr_t>(data) % tsize != 0)
            return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
        return with_functor(d, p, [&](auto f) -> rocrand_status { return run(f, data, n, tsize); });
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

private:
    template<class F>
    rocrand_status run(const F& f, void* data, size_t n, size_t tsize)
    {
        constexpr unsigned iw   = F::iw;
        constexpr unsigned ow   = F::ow;
        constexpr uint32_t full = kMtThreads * (kMtSlots / iw);
        const uintptr_t    addr = reinterpret_cast<uintptr_t>(data);
        const size_t       mis  = (ow - addr / tsize % ow) % ow;
        MtArgs             a;
        a.arena = m_arena;
        a.head  = static_cast<uint32_t>(n < mis ? n : mis);
        a.tail  = static_cast<uint32_t>((n - a.head) % ow);
        a.vec_n = (n - a.head) / ow;
        a.total = a.vec_n + ((a.head > 0 || a.tail > 0) ? 1 : 0);
        a.n     = n;
        a.data  = static_cast<unsigned char*>(data);
        a.vec   = a.data + mis * tsize;
        a.full  = full;
        // mt19937.hpp:957-971: after a change of input width, continue at the next slot
        // group no earlier call has read
        if(m_prev_iw != iw && m_start > 0)
        {
            const uint32_t used = (m_start + kMtThreads - 1) / kMtThreads * m_prev_iw;
            m_start             = (used + iw - 1) / iw * kMtThreads;
            if(m_start >= full)
                m_start = 0;
        }
        a.start       = m_start;
        a.twist_first = m_start == 0 ? 1u : 0u;
        a.rounds      = a.total == 0 ? 0u
                                     : static_cast<uint32_t>((m_start + a.total - 1) / full + 1);
        if(a.total > 0 && m_host_exec)
        {
            mt_fill_host(a, f, m_hstate.data());
        }
        else if(a.total > 0)
        {
            const size_t smem = mt_fill_smem(f);
            mt_fill<F><<<kMtThreads / kMtBlock, kMtBlock, smem, m_stream>>>(a, f);
            const rocrand_status st = launch_status();
            if(st != ROCRAND_STATUS_SUCCESS)
                return st;
        }
        m_start   = static_cast<uint32_t>((m_start + a.total) % full);
        m_prev_iw = iw;
        return ROCRAND_STATUS_SUCCESS;
    }

    uint32_t* m_arena   = nullptr;
    uint32_t  m_start   = 0;
    uint32_t  m_prev_iw = 0;
    // generator states of the CPU path, in word order (generator e at [e * 624])
    std::vector<uint32_t> m_hstate;
};

} // namespace

rocrand_generator_base_type* make_mt19937()
{
    return new Mt19937Generator();
}

} // namespace rb200
