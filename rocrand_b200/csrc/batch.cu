// batch.cu -- batched fill: thousands of generate requests in one persistent launch.
//
// Every request reproduces one plain call bit for bit: a Philox4x32-10, XORWOW, MRG32k3a or
// Sobol32 generator (fresh from a seed and offset, or a resident state owned by the
// server) and one of uint / uniform fp32 / uniform fp64 / normal fp32 / Poisson.  The host
// lays each request out as its plain call would (head, 16-byte or ow-vectors, tail),
// assigns it tiles, and uploads the descriptor table once; the kernel's blocks then take
// tiles from a global counter until none is left, so small and large requests, cheap
// (Philox) and seeding-heavy (a fresh XORWOW generator jumps each engine it uses to its
// subsequence) ones balance across the 148 SMs in one launch.
//   * Philox tile: a run of 16-byte vectors, vector j from stream position
//     4j + (j % 262144 == 0 ? start0 : head) (philox4x32_10.hpp:107-214);
//   * XORWOW / MRG32k3a tile: a run of engine slots; slot t drives engine (t + start) % E
//     and writes vectors t, t + E, ... (xorwow.hpp:63-161); a fresh engine is seeded here
//     from the request's base state with its subsequence jump;
//   * Sobol32 tile: a run of points of dimension 0, Gray-code steps within a thread and a
//     power-of-two leap-frog between a thread's runs (sobol.hpp:72-236).
#include "batch.hpp"

#include "common.hpp"
#include "dist.cuh"
#include "generators.hpp"
#include "launch.cuh"
#include "philox.cuh"
#include "poisson.hpp"
#include "sobol_dist.cuh"
#include "sobol_tables.hpp"
#include "jump_tables.hpp"
#include "stateful_engines.cuh"

#include <rocrand_b200.h>

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

namespace rb200
{

constexpr uint32_t kBatchBlock = 256;
constexpr uint32_t kBatchE     = kStatefulEngines;

struct BatchLaunch
{
    const BatchReq*     reqs;
    uint32_t            nreq;
    unsigned long long  tiles;
    unsigned long long* next;
    const uint32_t*     tile_req;     // request index of every tile
    const uint32_t*     xorwow_polys; // jump polynomials of the E engines
    const uint32_t*     xorwow_seqs;  // 2 x kXorwowSeqWords words per fresh XORWOW request
    const uint64_t*     mrg_tables;
    lr::Table           logf; // host-logf replay table (Sobol normal)
};

// ---- distribution functors of each engine family, built from a descriptor ----

template<class Body>
__device__ __forceinline__ void with_plain_functor(const BatchReq& r, Body&& body)
{
    switch(r.dist)
    {
        case BD_UINT: body(FnUint{}); break;
        case BD_FLOAT: body(FnFloat{}); break;
        case BD_DOUBLE: body(FnDouble{}); break;
        case BD_NORMAL_F: body(FnNormalF{r.mean, r.stddev}); break;
        default:
            if(r.huge)
                body(FnPoissonHuge{r.sqrt_lambda, r.lambda});
            else
                body(FnPoisson{r.thr, r.alias, r.tsize, r.toff});
            break;
    }
}

template<class Body>
__device__ __forceinline__ void with_mrg_functor(const BatchReq& r, Body&& body)
{
    using N = Mrg32k3aNorm;
    switch(r.dist)
    {
        case BD_UINT: body(FnMrgRemap<N, FnUint>{FnUint{}}); break;
        case BD_FLOAT: body(FnMrgFloat<N>{}); break;
        case BD_DOUBLE: body(FnMrgDouble<N>{}); break;
        case BD_NORMAL_F: body(FnMrgNormalF<N>{r.mean, r.stddev, false}); break;
        default:
            if(r.huge)
                body(FnMrgPoissonHuge<N>{r.sqrt_lambda, r.lambda});
            else
                body(FnMrgRemap<N, FnPoisson>{FnPoisson{r.thr, r.alias, r.tsize, r.toff}});
            break;
    }
}

// ---- tiles ----

template<class F>
__device__ __forceinline__ void philox_tile(const BatchReq& r, unsigned long long local, const F& f)
{
    const BatchPhilox&       p  = r.philox;
    const unsigned long long v0 = local * r.units;
    const unsigned long long v1 = v0 + r.units < r.vec_n ? v0 + r.units : r.vec_n;
    if(p.fast)
    {
        // two independent vectors per iteration so that the multiply chains interleave
        unsigned long long j = v0 + threadIdx.x;
        for(; j + blockDim.x < v1; j += 2 * blockDim.x)
        {
            const uint4 b0 = philox_block_lane(p.x0 + static_cast<uint32_t>(j), p.lane, p.keys);
            const uint4 b1 = philox_block_lane(p.x0 + static_cast<uint32_t>(j + blockDim.x), p.lane, p.keys);
            store16_cs(r.vec + j * 16, philox_vec(f, b0));
            store16_cs(r.vec + (j + blockDim.x) * 16, philox_vec(f, b1));
        }
        if(j < v1)
            store16_cs(r.vec + j * 16, philox_vec(f, philox_block_lane(p.x0 + static_cast<uint32_t>(j), p.lane, p.keys)));
    }
    else
    {
        for(unsigned long long j = v0 + threadIdx.x; j < v1; j += blockDim.x)
        {
            const uint32_t           adj = (j & (kPhiloxRefStride - 1)) == 0 ? p.start0 : p.head;
            const unsigned long long q   = p.s0 + adj + 4 * j;
            const uint4              c   = ctr_add(p.c0, q >> 2);
            const uint32_t           s   = static_cast<uint32_t>(q & 3);
            uint4                    b   = philox_block(c, p.keys);
            if(s != 0)
                b = interleave4(b, philox_block(ctr_add(c, 1), p.keys), s);
            store16_cs(r.vec + j * 16, philox_vec(f, b));
        }
    }
    if(local == 0 && threadIdx.x == 0 && (p.head > 0 || p.tail > 0))
    {
        PhiloxCall a;
        a.keys   = p.keys;
        a.c0     = p.c0;
        a.s0     = p.s0;
        a.head   = p.head;
        a.start0 = p.start0;
        a.tail   = p.tail;
        a.data   = r.data;
        a.vec    = r.vec;
        a.n      = r.n;
        a.vec_n  = r.vec_n;
        using T  = typename F::T;
        if(p.head > 0)
            philox_scalar_run(a, f, 0, reinterpret_cast<T*>(r.data), p.head);
        if(p.tail > 0)
        {
            const unsigned long long pos
                = 4 * r.vec_n + ((r.vec_n % kPhiloxRefStride) == 0 ? p.start0 : p.head);
            philox_scalar_run(a, f, pos, reinterpret_cast<T*>(r.data) + (r.n - p.tail), p.tail);
        }
    }
}

// Engine e of a fresh generator: the base state of its side of `start`, jumped e
// subsequences (as the plain generator's init kernels do); XORWOW from the window tables of
// the two bases, built by the block at the start of the tile.
template<class E>
__device__ __forceinline__ void seed_engine(const BatchReq& r, uint32_t e, E& eng, const BatchLaunch& L,
                                            const XorwowJumpTable* tables)
{
    const int which = e < r.start ? 1 : 0;
#pragma unroll
    for(int k = 0; k < 6; k++)
        eng.w[k] = r.base[which][k];
    if constexpr(std::is_same_v<E, XorwowEngine>)
    {
        xorwow_jump(tables[which], L.xorwow_polys, e, eng.w);
    }
    else
    {
        for(int p = 0; p < kJumpDigits; p++)
        {
            const uint32_t d = (e >> (2 * p)) & 3u;
            if(!d)
                continue;
            const uint64_t* t = L.mrg_tables + ((static_cast<size_t>(p) * 3 + (d - 1)) * 2) * 9;
            mod_apply(t, 4294967087ull, eng.w);
            mod_apply(t + 9, 4294944443ull, eng.w + 3);
        }
    }
}

template<class E, class F>
__device__ __forceinline__ void stateful_tile(const BatchReq& r, unsigned long long local, const F& f,
                                              const BatchLaunch& L, XorwowJumpTable* tables)
{
    using T               = typename F::T;
    constexpr unsigned VB = F::ow * sizeof(T);
    const bool         has_edge = F::ow > 1 && (r.head > 0 || r.tail > 0);
    const unsigned long long edge_slot = r.vec_n % kBatchE;
    const unsigned long long need = r.vec_n >= kBatchE ? kBatchE : r.vec_n + (has_edge ? 1 : 0);
    const unsigned long long t0   = local * r.units;
    const unsigned long long t1   = t0 + r.units < need ? t0 + r.units : need;
    if constexpr(std::is_same_v<E, XorwowEngine>)
    {
        if(r.arena == nullptr)
        {
            // slots t with t + start < E drive engines >= start (base 0), the rest base 1
            const uint32_t* seq = L.xorwow_seqs + static_cast<size_t>(r.xseq) * 2 * kXorwowSeqWords;
            if(t0 + r.start < kBatchE)
                xorwow_build_jump_table(tables[0], seq, threadIdx.x, blockDim.x);
            if(t1 - 1 + r.start >= kBatchE)
                xorwow_build_jump_table(tables[1], seq + kXorwowSeqWords, threadIdx.x, blockDim.x);
            __syncthreads();
        }
    }
    for(unsigned long long tb = t0; tb < t1; tb += blockDim.x)
    {
        const unsigned long long t     = tb + threadIdx.x;
        const bool               loops = t < t1 && t < r.vec_n;
        const bool               edges = t < t1 && has_edge && edge_slot == t;
        const uint32_t           e     = static_cast<uint32_t>((t + r.start) & (kBatchE - 1));
        E                        eng;
        if(r.arena)
        {
            if(!loops && !edges)
                continue;
#pragma unroll
            for(int k = 0; k < E::kWords; k++)
                eng.w[k] = r.arena[static_cast<size_t>(k) * kBatchE + e];
        }
        else
        {
            if(!loops && !edges)
                continue;
            seed_engine(r, e, eng, L, tables);
        }
        uint32_t           in[F::iw];
        T                  out[F::ow];
        unsigned long long j = t;
        for(; j < r.vec_n; j += kBatchE)
        {
#pragma unroll
            for(unsigned i = 0; i < F::iw; i++)
                in[i] = eng.next();
            f(in, out);
            store_small(r.vec + j * VB, out);
        }
        if(F::ow > 1 && j == r.vec_n)
        {
            T* data = reinterpret_cast<T*>(r.data);
            if(r.head > 0)
            {
                for(unsigned i = 0; i < F::iw; i++)
                    in[i] = eng.next();
                f(in, out);
                for(unsigned o = 0; o < r.head; o++)
                    data[o] = out[o];
            }
            if(r.tail > 0)
            {
                for(unsigned i = 0; i < F::iw; i++)
                    in[i] = eng.next();
                f(in, out);
                for(unsigned o = 0; o < r.tail; o++)
                    data[r.n - r.tail + o] = out[o];
            }
        }
        if(r.arena)
        {
#pragma unroll
            for(int k = 0; k < E::kWords; k++)
                r.arena[static_cast<size_t>(k) * kBatchE + e] = eng.w[k];
        }
    }
}

template<SobolKind K>
__device__ __forceinline__ void sobol_tile(const BatchReq& r, unsigned long long local, const lr::Table& logf)
{
    using T                   = typename SobolOut<K, uint32_t>::T;
    constexpr unsigned PPT    = sizeof(T) >= 4 ? 4u : 16u / sizeof(T);
    const uint32_t     stride = PPT * blockDim.x; // a power of two
    const uint32_t     lg     = __ffs(stride) - 1;
    const unsigned long long p0 = local * r.units;
    const unsigned long long p1 = p0 + r.units < r.n ? p0 + r.units : r.n;
    unsigned long long       p  = p0 + static_cast<unsigned long long>(threadIdx.x) * PPT;
    if(p >= p1)
        return;
    SobolParams sp;
    sp.mean_f      = r.mean;
    sp.std_f       = r.stddev;
    sp.cdf         = r.cdf;
    sp.size        = r.tsize;
    sp.offset      = r.toff;
    sp.lambda      = r.lambda;
    sp.sqrt_lambda = r.sqrt_lambda;
    sp.logf        = logf;
    const uint32_t* v   = r.sobol_v;
    T*              row = reinterpret_cast<T*>(r.data);
    // the engine starts at the 32-bit sum offset + p (sobol.hpp:191-196)
    uint32_t i = r.sobol_offset + static_cast<uint32_t>(p);
    uint32_t x = 0;
    {
        const uint32_t g = i ^ (i >> 1);
        for(int b = 0; b < 32; b++)
            if((g >> b) & 1u)
                x ^= __ldg(v + b);
    }
    const bool vec_ok = (reinterpret_cast<uintptr_t>(row) % (PPT * sizeof(T))) == 0;
    for(; p < p1; p += stride)
    {
        T        out[PPT];
        uint32_t xx = x, ii = i;
#pragma unroll
        for(unsigned k = 0; k < PPT; k++)
        {
            out[k] = sobol_apply<K, uint32_t>(xx, sp, r.cdf);
            xx ^= __ldg(v + rzb(ii));
            ii++;
        }
        if(vec_ok && p + PPT <= p1)
        {
            constexpr unsigned VB = PPT * sizeof(T);
            uint4              w[VB / 16];
            memcpy(w, out, VB);
#pragma unroll
            for(unsigned k = 0; k < VB / 16; k++)
                __stcs(reinterpret_cast<uint4*>(row + p) + k, w[k]);
        }
        else
        {
            for(unsigned k = 0; k < PPT && p + k < p1; k++)
                row[p + k] = out[k];
        }
        x ^= __ldg(v + lg - 1);
        x ^= __ldg(v + rzb(i | (stride - 1)));
        i += stride;
    }
}

__global__ void __launch_bounds__(kBatchBlock, 4) batch_fill(BatchLaunch L)
{
    // Tiles come from a global counter; thread 0 keeps the next two in flight so that their
    // counter and request-map reads overlap the current tile's work: while tile t runs, the
    // request of the next tile and the index of the one after it are being fetched.
    __shared__ unsigned long long s_tile, s_next;
    __shared__ uint32_t           s_req;
    __shared__ XorwowJumpTable    s_xorwow[2]; // fresh XORWOW tiles: window tables of the bases
    if(threadIdx.x == 0)
    {
        const unsigned long long t = atomicAdd(L.next, 1ull);
        s_tile                     = t;
        s_req                      = t < L.tiles ? L.tile_req[t] : 0u;
        s_next                     = atomicAdd(L.next, 1ull);
    }
    __syncthreads();
    for(;;)
    {
        const unsigned long long t = s_tile;
        if(t >= L.tiles)
            return;
        unsigned long long next = 0, after = 0;
        uint32_t           next_req = 0;
        if(threadIdx.x == 0)
        {
            next = s_next;
            if(next < L.tiles)
            {
                next_req = L.tile_req[next];
                after    = atomicAdd(L.next, 1ull);
            }
            else
            {
                after = next;
            }
        }
        const BatchReq&          r     = L.reqs[s_req];
        const unsigned long long local = t - r.tile0;
        switch(r.kind)
        {
            case BK_PHILOX:
                with_plain_functor(r, [&](auto f) { philox_tile(r, local, f); });
                break;
            case BK_XORWOW:
                with_plain_functor(r, [&](auto f) { stateful_tile<XorwowEngine>(r, local, f, L, s_xorwow); });
                break;
            case BK_MRG32K3A:
                with_mrg_functor(r, [&](auto f) { stateful_tile<Mrg32k3aEngine>(r, local, f, L, s_xorwow); });
                break;
            default:
                switch(r.dist)
                {
                    case BD_UINT: sobol_tile<SobolKind::UINT>(r, local, L.logf); break;
                    case BD_FLOAT: sobol_tile<SobolKind::FLOAT>(r, local, L.logf); break;
                    case BD_DOUBLE: sobol_tile<SobolKind::DOUBLE>(r, local, L.logf); break;
                    case BD_NORMAL_F: sobol_tile<SobolKind::NORMAL_F>(r, local, L.logf); break;
                    default:
                        if(r.huge)
                            sobol_tile<SobolKind::POISSON_HUGE>(r, local, L.logf);
                        else
                            sobol_tile<SobolKind::POISSON>(r, local, L.logf);
                        break;
                }
                break;
        }
        __syncthreads();
        if(threadIdx.x == 0)
        {
            s_tile = next;
            s_req  = next_req;
            s_next = after;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Host side.

BatchTuning& batch_tuning()
{
    static BatchTuning t = [] {
        BatchTuning d{};
        for(uint32_t k = 0; k < BK_COUNT; k++)
            for(uint32_t dd = 0; dd < BD_COUNT; dd++)
            {
                d.units[k][dd] = k == BK_PHILOX ? 4096u : (k == BK_SOBOL32 ? 8192u : (k == BK_XORWOW ? 1024u : 256u));
                // serving: smaller tiles keep small requests' latency low and balance mixes
                d.serve_units[k][dd] = k == BK_PHILOX ? 2048u : (k == BK_SOBOL32 ? 8192u : 256u);
            }
        d.blocks_per_sm = 0; // 0: occupancy
        return d;
    }();
    return t;
}

uint32_t batch_elem_size(uint32_t dist)
{
    return dist == BD_DOUBLE ? 8u : 4u;
}

// Poisson tables shared by all batches, one per (device, lambda, cdf).
static rocrand_status poisson_for(double lambda, bool cdf, cudaStream_t stream, DistParams& p)
{
    static std::mutex                                                   mu;
    static std::map<std::tuple<int, double, bool>, std::unique_ptr<PoissonCache>> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto&      slot  = cache[std::make_tuple(device_info().device, lambda, cdf)];
    const bool fresh = !slot;
    if(fresh)
        slot.reset(new PoissonCache());
    rocrand_status st = slot->get(lambda, stream, cdf, p);
    // batches on every stream read the table: a new one is uploaded before anyone uses it
    // (once per lambda; plans and the server build descriptors outside any stream capture)
    if(st == ROCRAND_STATUS_SUCCESS && fresh && !p.huge && cudaStreamSynchronize(stream) != cudaSuccess)
        st = ROCRAND_STATUS_LAUNCH_FAILURE;
    return st;
}

rocrand_status batch_set_dist(BatchReq& r, uint32_t dist, double p0, double p1, cudaStream_t stream)
{
    if(dist >= BD_COUNT)
        return ROCRAND_STATUS_TYPE_ERROR;
    r.dist   = dist;
    r.mean   = static_cast<float>(p0);
    r.stddev = static_cast<float>(p1);
    r.prob   = nullptr;
    r.thr    = nullptr;
    r.alias  = nullptr;
    r.cdf    = nullptr;
    r.tsize = r.toff = r.huge = 0;
    r.lambda = r.sqrt_lambda = 0.0;
    if(dist == BD_POISSON)
    {
        if(!(p0 > 0.0))
            return ROCRAND_STATUS_OUT_OF_RANGE;
        DistParams     dp;
        rocrand_status st = poisson_for(p0, r.kind == BK_SOBOL32, stream, dp);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        r.prob        = dp.prob;
        r.thr         = dp.thr;
        r.alias       = dp.alias;
        r.cdf         = dp.cdf;
        r.tsize       = dp.size;
        r.toff        = dp.offset;
        r.huge        = dp.huge;
        r.lambda      = dp.lambda;
        r.sqrt_lambda = dp.sqrt_lambda;
    }
    return ROCRAND_STATUS_SUCCESS;
}

// Inputs and outputs per distribution call of each family (functors of dist.cuh).
void batch_widths(uint32_t kind, uint32_t dist, unsigned& iw, unsigned& ow)
{
    iw = 1;
    ow = 1;
    if(dist == BD_NORMAL_F)
        iw = ow = 2;
    else if(dist == BD_DOUBLE && kind != BK_MRG32K3A)
        iw = 2; // MRG doubles come from one output (FnMrgDouble)
}

rocrand_status batch_layout(BatchReq& r, void* output, size_t n)
{
    const uint32_t  tsize = batch_elem_size(r.dist);
    const uintptr_t addr  = reinterpret_cast<uintptr_t>(output);
    if(output == nullptr || addr % tsize != 0)
        return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
    r.data = static_cast<unsigned char*>(output);
    r.n    = n;
    unsigned iw, ow;
    batch_widths(r.kind, r.dist, iw, ow);
    if(r.kind == BK_PHILOX)
    {
        const unsigned fow = (4 / iw) * ow; // elements per 16-byte vector
        const size_t   mis = (fow - addr / tsize % fow) % fow;
        r.philox.head      = static_cast<uint32_t>(n < mis ? n : mis);
        r.philox.tail      = static_cast<uint32_t>((n - r.philox.head) % fow);
        r.vec_n            = (n - r.philox.head) / fow;
        r.philox.start0    = r.philox.head > 0 ? (r.philox.head + ow - 1) / ow * iw : 0;
        r.vec              = r.data + mis * tsize;
        r.head             = r.philox.head;
        r.tail             = r.philox.tail;
        r.philox.fast      = 0;
        if(r.philox.start0 == r.philox.head && ((r.philox.s0 + r.philox.head) & 3u) == 0)
        {
            const uint4 cbase = ctr_add(r.philox.c0, (r.philox.s0 + r.philox.head) >> 2);
            if(static_cast<unsigned long long>(cbase.x) + r.vec_n <= (1ull << 32))
            {
                r.philox.fast = 1;
                r.philox.x0   = cbase.x;
                r.philox.lane = philox_lane(cbase, r.philox.keys);
            }
        }
    }
    else if(r.kind == BK_SOBOL32)
    {
        r.vec_n = n;
        r.vec   = r.data;
        r.head = r.tail = 0;
    }
    else
    {
        const size_t mis = (ow - addr / tsize % ow) % ow;
        r.head           = static_cast<uint32_t>(n < mis ? n : mis);
        r.tail           = static_cast<uint32_t>((n - r.head) % ow);
        r.vec_n          = (n - r.head) / ow;
        r.vec            = r.data + mis * tsize;
    }
    return ROCRAND_STATUS_SUCCESS;
}

static unsigned long long tiles_of(const BatchReq& r)
{
    if(r.n == 0)
        return 0;
    const unsigned long long u = r.units;
    if(r.kind == BK_PHILOX)
        return r.vec_n == 0 ? 1 : (r.vec_n + u - 1) / u;
    if(r.kind == BK_SOBOL32)
        return (r.n + u - 1) / u;
    unsigned iw, ow;
    batch_widths(r.kind, r.dist, iw, ow);
    const bool edge = ow > 1 && (r.head > 0 || r.tail > 0);
    const unsigned long long need
        = r.vec_n >= kBatchE ? kBatchE : r.vec_n + (edge ? 1 : 0);
    return (need + u - 1) / u;
}

BatchPlan::~BatchPlan()
{
    if(m_exec)
        cudaGraphExecDestroy(m_exec);
    if(m_staged)
    {
        cudaEventSynchronize(m_staged);
        cudaEventDestroy(m_staged);
    }
    cudaFreeHost(h_stage);
    cudaFree(d_reqs);
    cudaFree(d_seq);
    cudaFree(d_tile_req);
}

rocrand_status BatchPlan::build(const void* requests, size_t count, cudaStream_t stream)
{
    const auto* q = static_cast<const rocrand_b200_request*>(requests);
    m_reqs.clear();
    m_seq.clear();
    m_reqs.reserve(count);
    for(size_t i = 0; i < count; i++)
    {
        const rocrand_b200_request& u = q[i];
        BatchReq                    r{};
        switch(u.rng_type)
        {
            case ROCRAND_RNG_PSEUDO_PHILOX4_32_10:
            {
                r.kind = BK_PHILOX;
                CounterPos pos;
                pos.advance(u.offset);
                r.philox.keys = philox_keys(u.seed);
                r.philox.c0   = pos.counter;
                r.philox.s0   = pos.sub;
                break;
            }
            case ROCRAND_RNG_PSEUDO_DEFAULT:
            case ROCRAND_RNG_PSEUDO_XORWOW:
            case ROCRAND_RNG_PSEUDO_MRG32K3A:
            {
                const bool xw = u.rng_type != ROCRAND_RNG_PSEUDO_MRG32K3A;
                r.kind        = xw ? BK_XORWOW : BK_MRG32K3A;
                const StatefulBases b
                    = stateful_bases(xw ? StatefulFamily::XORWOW : StatefulFamily::MRG32K3A, u.seed,
                                     u.offset);
                memcpy(r.base, b.base, sizeof(r.base));
                r.start = b.start;
                r.arena = nullptr;
                if(xw)
                {
                    r.xseq = static_cast<uint32_t>(m_seq.size() / (2 * kXorwowSeqWords));
                    m_seq.resize(m_seq.size() + 2 * kXorwowSeqWords);
                    uint32_t* seq = m_seq.data() + m_seq.size() - 2 * kXorwowSeqWords;
                    xorwow_word_sequence(r.base[0], seq);
                    xorwow_word_sequence(r.base[1], seq + kXorwowSeqWords);
                }
                break;
            }
            case ROCRAND_RNG_QUASI_DEFAULT:
            case ROCRAND_RNG_QUASI_SOBOL32:
            {
                r.kind         = BK_SOBOL32;
                r.sobol_offset = static_cast<uint32_t>(u.offset); // 32-bit counter (sobol.hpp:604)
                r.sobol_v      = static_cast<const uint32_t*>(sobol_device_vectors(false, false));
                if(r.sobol_v == nullptr)
                    return ROCRAND_STATUS_ALLOCATION_FAILED;
                break;
            }
            default: return ROCRAND_STATUS_TYPE_ERROR;
        }
        rocrand_status st = batch_set_dist(r, static_cast<uint32_t>(u.distribution), u.param0,
                                           u.param1, stream);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        st = batch_layout(r, u.output, u.n);
        if(st != ROCRAND_STATUS_SUCCESS && u.n > 0)
            return st;
        if(u.n == 0)
            continue;
        m_reqs.push_back(r);
    }
    return ROCRAND_STATUS_SUCCESS;
}

rocrand_status BatchPlan::reserve(size_t reqs, size_t tiles)
{
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    if(reqs > m_cap || dev != m_device)
    {
        cudaFree(d_reqs);
        d_reqs = nullptr;
        m_cap  = 0;
        if(cudaMalloc(&d_reqs, sizeof(BatchReq) * reqs + 256) != cudaSuccess)
        {
            d_reqs = nullptr;
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        }
        m_cap    = reqs;
        m_device = dev;
        if(m_exec)
        {
            cudaGraphExecDestroy(m_exec);
            m_exec = nullptr;
        }
    }
    if(tiles > m_tile_cap)
    {
        cudaFree(d_tile_req);
        d_tile_req = nullptr;
        m_tile_cap = 0;
        if(cudaMalloc(&d_tile_req, sizeof(uint32_t) * tiles) != cudaSuccess)
        {
            d_tile_req = nullptr;
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        }
        m_tile_cap = tiles;
    }
    const size_t stage = sizeof(uint32_t) * tiles + sizeof(BatchReq) * reqs + 32;
    if(stage > m_stage_cap)
    {
        cudaFreeHost(h_stage);
        h_stage     = nullptr;
        m_stage_cap = 0;
        if(cudaHostAlloc(reinterpret_cast<void**>(&h_stage), stage, cudaHostAllocDefault) != cudaSuccess)
        {
            h_stage = nullptr;
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        }
        m_stage_cap = stage;
    }
    if(m_staged == nullptr && cudaEventCreateWithFlags(&m_staged, cudaEventDisableTiming) != cudaSuccess)
    {
        m_staged = nullptr;
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
    // load the kernel and upload the per-device jump tables now (a module loads lazily at a
    // kernel's first use, tens of ms, and the tables are copied on first use; both would
    // otherwise land on the first batch)
    cudaFuncAttributes attr;
    if(cudaFuncGetAttributes(&attr, batch_fill) != cudaSuccess)
        return ROCRAND_STATUS_LAUNCH_FAILURE;
    if(stateful_xorwow_jump_polys() == nullptr || stateful_digit_tables(StatefulFamily::MRG32K3A) == nullptr)
        return ROCRAND_STATUS_ALLOCATION_FAILED;
    return ROCRAND_STATUS_SUCCESS;
}

rocrand_status BatchPlan::upload(cudaStream_t stream)
{
    const BatchTuning& tune = batch_tuning();
    m_tiles                 = 0;
    m_bytes                 = 0;
    m_tile_req.clear();
    for(size_t i = 0; i < m_reqs.size(); i++)
    {
        BatchReq& r = m_reqs[i];
        r.units     = m_serving ? tune.serve_units[r.kind][r.dist] : tune.units[r.kind][r.dist];
        r.tile0     = m_tiles;
        m_tiles += tiles_of(r);
        m_bytes += r.n * batch_elem_size(r.dist);
        m_tile_req.resize(m_tiles, static_cast<uint32_t>(i));
    }
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    // Device tables grow geometrically: cudaFree synchronises the whole device, which would
    // serialise the server's streams if a table were resized for every batch.
    if(m_reqs.size() > m_cap || dev != m_device)
    {
        cudaFree(d_reqs);
        d_reqs = nullptr;
        m_cap  = std::max<size_t>({m_reqs.size(), 2 * m_cap, 256});
        // descriptors followed by the tile counter
        if(cudaMalloc(&d_reqs, sizeof(BatchReq) * m_cap + 256) != cudaSuccess)
        {
            d_reqs = nullptr;
            m_cap  = 0;
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        }
        m_device = dev;
        if(m_exec)
        {
            cudaGraphExecDestroy(m_exec);
            m_exec = nullptr;
        }
    }
    if(m_seq.size() > m_seq_cap)
    {
        cudaFree(d_seq);
        d_seq = nullptr;
        const size_t cap = std::max<size_t>({m_seq.size(), 2 * m_seq_cap, 2 * kXorwowSeqWords * 64});
        if(cudaMalloc(&d_seq, sizeof(uint32_t) * cap) != cudaSuccess)
        {
            d_seq     = nullptr;
            m_seq_cap = 0;
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        }
        m_seq_cap = cap;
        if(m_exec)
        {
            cudaGraphExecDestroy(m_exec);
            m_exec = nullptr;
        }
    }
    if(m_tile_req.size() > m_tile_cap)
    {
        cudaFree(d_tile_req);
        d_tile_req = nullptr;
        const size_t cap = std::max<size_t>({m_tile_req.size(), 2 * m_tile_cap, size_t(1) << 16});
        if(cudaMalloc(&d_tile_req, sizeof(uint32_t) * cap) != cudaSuccess)
        {
            d_tile_req = nullptr;
            m_tile_cap = 0;
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        }
        m_tile_cap = cap;
        if(m_exec)
        {
            cudaGraphExecDestroy(m_exec);
            m_exec = nullptr;
        }
    }
    d_next = reinterpret_cast<unsigned long long*>(reinterpret_cast<unsigned char*>(d_reqs)
                                                   + sizeof(BatchReq) * m_cap);
    // the three tables go through one pinned buffer, which the previous upload's copies must
    // have read before it is refilled (immediate in the server: a plan's last batch is done)
    auto         up16   = [](size_t b) { return (b + 15) / 16 * 16; };
    const size_t b_tile = sizeof(uint32_t) * m_tile_req.size();
    const size_t b_seq  = sizeof(uint32_t) * m_seq.size();
    const size_t b_reqs = sizeof(BatchReq) * m_reqs.size();
    const size_t total  = up16(b_tile) + up16(b_seq) + b_reqs;
    if(total == 0)
        return ROCRAND_STATUS_SUCCESS;
    if(m_staged == nullptr && cudaEventCreateWithFlags(&m_staged, cudaEventDisableTiming) != cudaSuccess)
    {
        m_staged = nullptr;
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
    if(cudaEventSynchronize(m_staged) != cudaSuccess)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    if(total > m_stage_cap)
    {
        const size_t cap = std::max<size_t>({total, 2 * m_stage_cap, size_t(1) << 20});
        cudaFreeHost(h_stage);
        h_stage     = nullptr;
        m_stage_cap = 0;
        if(cudaHostAlloc(reinterpret_cast<void**>(&h_stage), cap, cudaHostAllocDefault) != cudaSuccess)
        {
            h_stage = nullptr;
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        }
        m_stage_cap = cap;
    }
    unsigned char* seq  = h_stage + up16(b_tile);
    unsigned char* reqs = seq + up16(b_seq);
    if(b_tile)
        std::memcpy(h_stage, m_tile_req.data(), b_tile);
    if(b_seq)
        std::memcpy(seq, m_seq.data(), b_seq);
    if(b_reqs)
        std::memcpy(reqs, m_reqs.data(), b_reqs);
    if((b_tile && cudaMemcpyAsync(d_tile_req, h_stage, b_tile, cudaMemcpyHostToDevice, stream) != cudaSuccess)
       || (b_seq && cudaMemcpyAsync(d_seq, seq, b_seq, cudaMemcpyHostToDevice, stream) != cudaSuccess)
       || (b_reqs && cudaMemcpyAsync(d_reqs, reqs, b_reqs, cudaMemcpyHostToDevice, stream) != cudaSuccess)
       || cudaEventRecord(m_staged, stream) != cudaSuccess)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    return ROCRAND_STATUS_SUCCESS;
}

static unsigned batch_grid()
{
    static std::atomic<int> occ_cache{0}; // computed once; concurrent first calls agree
    int                     occ = occ_cache.load(std::memory_order_relaxed);
    if(occ == 0)
    {
        if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_fill, kBatchBlock, 0) != cudaSuccess
           || occ < 1)
            occ = 1;
        occ_cache.store(occ, std::memory_order_relaxed);
    }
    const uint32_t per = batch_tuning().blocks_per_sm;
    const unsigned b   = per > 0 && per < static_cast<uint32_t>(occ) ? per : static_cast<unsigned>(occ);
    return b * static_cast<unsigned>(device_info().sm_count);
}

rocrand_status BatchPlan::launch(cudaStream_t stream)
{
    if(m_tiles == 0)
        return ROCRAND_STATUS_SUCCESS;
    if(cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), stream) != cudaSuccess)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    BatchLaunch L;
    L.reqs          = d_reqs;
    L.nreq          = static_cast<uint32_t>(m_reqs.size());
    L.tiles         = m_tiles;
    L.next          = d_next;
    L.tile_req      = d_tile_req;
    L.xorwow_polys  = stateful_xorwow_jump_polys();
    L.xorwow_seqs   = d_seq;
    L.mrg_tables    = static_cast<const uint64_t*>(stateful_digit_tables(StatefulFamily::MRG32K3A));
    if(L.xorwow_polys == nullptr || L.mrg_tables == nullptr || !logf_replay_device(L.logf))
        return ROCRAND_STATUS_ALLOCATION_FAILED;
    const unsigned long long want = m_tiles;
    unsigned                 grid = batch_grid();
    if(want < grid)
        grid = static_cast<unsigned>(want);
    batch_fill<<<grid, kBatchBlock, 0, stream>>>(L);
    return launch_status();
}

rocrand_status BatchPlan::replay(cudaStream_t stream)
{
    if(m_tiles == 0)
        return ROCRAND_STATUS_SUCCESS;
    if(m_exec == nullptr)
    {
        // tables and the grid are resolved before capture (their first use uploads/queries)
        (void)batch_grid();
        lr::Table lt;
        if(stateful_xorwow_jump_polys() == nullptr
           || stateful_digit_tables(StatefulFamily::MRG32K3A) == nullptr || !logf_replay_device(lt))
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        cudaStream_t cap = nullptr;
        if(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        cudaGraph_t    graph = nullptr;
        rocrand_status st    = ROCRAND_STATUS_SUCCESS;
        if(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            st = ROCRAND_STATUS_INTERNAL_ERROR;
        else
        {
            st = launch(cap);
            if(cudaStreamEndCapture(cap, &graph) != cudaSuccess)
                st = ROCRAND_STATUS_INTERNAL_ERROR;
        }
        if(st == ROCRAND_STATUS_SUCCESS
           && cudaGraphInstantiate(&m_exec, graph, 0) != cudaSuccess)
        {
            m_exec = nullptr;
            st     = ROCRAND_STATUS_INTERNAL_ERROR;
        }
        if(graph)
            cudaGraphDestroy(graph);
        cudaStreamDestroy(cap);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
    }
    return cudaGraphLaunch(m_exec, stream) == cudaSuccess ? ROCRAND_STATUS_SUCCESS
                                                           : ROCRAND_STATUS_LAUNCH_FAILURE;
}

} // namespace rb200

using namespace rb200;

struct rocrand_b200_batch_plan_st
{
    BatchPlan plan;
};

extern "C" rocrand_status ROCRANDAPI rocrand_b200_generate_batch(const rocrand_b200_request* requests,
                                                                 size_t count, cudaStream_t stream)
{
    if(requests == nullptr && count > 0)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        BatchPlan      p;
        rocrand_status st = p.build(requests, count, stream);
        if(st == ROCRAND_STATUS_SUCCESS)
            st = p.upload(stream);
        if(st == ROCRAND_STATUS_SUCCESS)
            st = p.launch(stream);
        // the plan's device table is freed when it goes out of scope: wait for the launch
        if(cudaStreamSynchronize(stream) != cudaSuccess && st == ROCRAND_STATUS_SUCCESS)
            st = ROCRAND_STATUS_LAUNCH_FAILURE;
        return st;
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_create_batch_plan(rocrand_b200_batch_plan* plan,
                                                                    const rocrand_b200_request* requests,
                                                                    size_t count, cudaStream_t stream)
{
    if(plan == nullptr || (requests == nullptr && count > 0))
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        auto           p  = std::make_unique<rocrand_b200_batch_plan_st>();
        rocrand_status st = p->plan.build(requests, count, stream);
        if(st == ROCRAND_STATUS_SUCCESS)
            st = p->plan.upload(stream);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        *plan = p.release();
        return ROCRAND_STATUS_SUCCESS;
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_execute_batch_plan(rocrand_b200_batch_plan plan,
                                                                     int use_graph, cudaStream_t stream)
{
    if(plan == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    try
    {
        return use_graph ? plan->plan.replay(stream) : plan->plan.launch(stream);
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_destroy_batch_plan(rocrand_b200_batch_plan plan)
{
    if(plan == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    cudaDeviceSynchronize();
    delete plan;
    return ROCRAND_STATUS_SUCCESS;
}

namespace
{

int batch_kind_of(rocrand_rng_type t)
{
    switch(t)
    {
        case ROCRAND_RNG_PSEUDO_PHILOX4_32_10: return BK_PHILOX;
        case ROCRAND_RNG_PSEUDO_DEFAULT:
        case ROCRAND_RNG_PSEUDO_XORWOW: return BK_XORWOW;
        case ROCRAND_RNG_PSEUDO_MRG32K3A: return BK_MRG32K3A;
        case ROCRAND_RNG_QUASI_DEFAULT:
        case ROCRAND_RNG_QUASI_SOBOL32: return BK_SOBOL32;
        default: return -1;
    }
}

// Device time of one launch of `plan`, best of `reps`.
float time_plan(BatchPlan& plan, cudaStream_t stream, int reps)
{
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    for(int k = 0; k < reps; k++)
    {
        cudaEventRecord(a, stream);
        plan.launch(stream);
        cudaEventRecord(b, stream);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        best = ms < best ? ms : best;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

} // namespace

extern "C" rocrand_status ROCRANDAPI rocrand_b200_autotune_batch(cudaStream_t stream)
{
    try
    {
        // synthetic batch per pair: 48 fresh generators x 2^20 values (sizes of the
        // log-uniform request mix's middle), outputs in one scratch buffer
        constexpr size_t kReq = 48, kN = size_t(1) << 20;
        void*            scratch = nullptr;
        if(cudaMalloc(&scratch, kReq * kN * 8) != cudaSuccess)
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        const rocrand_rng_type types[BK_COUNT] = {ROCRAND_RNG_PSEUDO_PHILOX4_32_10,
                                                  ROCRAND_RNG_PSEUDO_XORWOW,
                                                  ROCRAND_RNG_PSEUDO_MRG32K3A,
                                                  ROCRAND_RNG_QUASI_SOBOL32};
        const std::vector<uint32_t> cand[BK_COUNT]
            = {{1024, 2048, 4096, 8192, 16384}, {256, 512, 1024, 2048, 4096}, {128, 256, 512, 1024, 2048},
               {2048, 4096, 8192, 16384, 32768}};
        BatchTuning&   tune = batch_tuning();
        rocrand_status st   = ROCRAND_STATUS_SUCCESS;
        for(uint32_t k = 0; k < BK_COUNT && st == ROCRAND_STATUS_SUCCESS; k++)
        {
            for(uint32_t d = 0; d < BD_COUNT && st == ROCRAND_STATUS_SUCCESS; d++)
            {
                std::vector<rocrand_b200_request> reqs(kReq);
                for(size_t i = 0; i < kReq; i++)
                {
                    rocrand_b200_request& q = reqs[i];
                    q.rng_type              = types[k];
                    q.distribution          = static_cast<rocrand_b200_distribution>(d);
                    q.seed                  = 0x9e3779b97f4a7c15ull * (i + 1);
                    q.offset                = 0;
                    q.param0                = d == BD_POISSON ? 4.0 : 0.0;
                    q.param1                = 1.0;
                    q.output                = static_cast<unsigned char*>(scratch) + i * kN * 8;
                    q.n                     = kN;
                }
                BatchPlan plan;
                st = plan.build(reqs.data(), reqs.size(), stream);
                if(st != ROCRAND_STATUS_SUCCESS)
                    break;
                const uint32_t keep = tune.units[k][d];
                uint32_t       best_u = keep;
                float          best_t = 1e30f;
                for(uint32_t u : cand[k])
                {
                    tune.units[k][d] = u;
                    st               = plan.upload(stream);
                    if(st != ROCRAND_STATUS_SUCCESS)
                        break;
                    time_plan(plan, stream, 1); // warm-up (first use uploads tables)
                    const float t = time_plan(plan, stream, 3);
                    if(t < best_t)
                    {
                        best_t = t;
                        best_u = u;
                    }
                }
                tune.units[k][d] = st == ROCRAND_STATUS_SUCCESS ? best_u : keep;
            }
        }
        cudaStreamSynchronize(stream);
        cudaFree(scratch);
        return st;
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_get_batch_tile(rocrand_rng_type          rng_type,
                                                                 rocrand_b200_distribution distribution,
                                                                 unsigned int*             units)
{
    const int k = batch_kind_of(rng_type);
    if(units == nullptr || k < 0 || static_cast<uint32_t>(distribution) >= BD_COUNT)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    *units = batch_tuning().units[k][distribution];
    return ROCRAND_STATUS_SUCCESS;
}
