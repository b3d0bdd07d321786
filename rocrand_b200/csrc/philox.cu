// philox.cu -- Philox4x32-10 generator: host object and fused sm_100a kernels.
//
// Output contract (what the reference's generate_philox, library/src/rng/philox4x32_10.hpp
// :107-214, produces on its default 1024x256 grid), restated position by position so any
// grid gives identical bytes:
//   * the output is split into a head of `head` elements (up to the first 16-byte
//     boundary), vec_n 16-byte vectors and a tail;
//   * vector j holds the distribution applied to the 4 stream values starting at
//     p(j) = 4*j + (j % 262144 == 0 ? start0 : head), where start0 = ceil(head/ow)*iw is
//     how far the head moved thread 0 of the reference grid;
//   * the head is produced sequentially from stream position 0, the tail sequentially
//     from p(vec_n);
//   * positions are relative to the generator's engine position, which advances by
//     ceil(n/ow)*iw per call (philox4x32_10.hpp:349-354).
// The common case (start0 == head and a block-aligned start) needs one Philox block per
// vector; otherwise a vector straddles two blocks.
#include "common.hpp"
#include "counter_engines.cuh"
#include "dist.cuh"
#include "generators.hpp"
#include "launch.cuh"
#include "batch.hpp"
#include "host_exec.hpp"
#include "philox.cuh"
#include "poisson.hpp"

#include <cstring>

namespace rb200
{

// kAligned: start0 == head and (s0 + head) % 4 == 0, so vector j is exactly block
// c0 + (s0 + head)/4 + j.
template<class F, bool kAligned>
__global__ void __launch_bounds__(kBlock) philox_fill(PhiloxCall a, F f)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const F g = stage_table(f, smem);

    const unsigned long long tid    = static_cast<unsigned long long>(blockIdx.x) * kBlock + threadIdx.x;
    const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * kBlock;

    if(kAligned)
    {
        const uint4 cbase = ctr_add(a.c0, (a.s0 + a.head) >> 2);
        for(unsigned long long j = tid; j < a.vec_n; j += stride)
        {
            const uint4 b = philox_block(ctr_add(cbase, j), a.keys);
            store16_cs(a.vec + j * 16, philox_vec(g, b));
        }
    }
    else
    {
        for(unsigned long long j = tid; j < a.vec_n; j += stride)
        {
            const uint32_t adj = (j & (kPhiloxRefStride - 1)) == 0 ? a.start0 : a.head;
            const unsigned long long q = a.s0 + adj + 4 * j;
            const uint4 c  = ctr_add(a.c0, q >> 2);
            const uint32_t s = static_cast<uint32_t>(q & 3);
            uint4 b = philox_block(c, a.keys);
            if(s != 0)
                b = interleave4(b, philox_block(ctr_add(c, 1), a.keys), s);
            store16_cs(a.vec + j * 16, philox_vec(g, b));
        }
    }

    if(tid == 0)
    {
        using T = typename F::T;
        if(a.head > 0)
            philox_scalar_run(a, g, 0, reinterpret_cast<T*>(a.data), a.head);
        if(a.tail > 0)
        {
            const unsigned long long pos
                = 4 * a.vec_n + ((a.vec_n % kPhiloxRefStride) == 0 ? a.start0 : a.head);
            philox_scalar_run(a, g, pos, reinterpret_cast<T*>(a.data) + (a.n - a.tail), a.tail);
        }
    }
}

// Fast path: aligned vectors whose counters (x0 + j, y, z, w) share the upper words for the
// whole launch (x0 + vec_n <= 2^32, checked by the host).  Each thread produces two
// independent vectors per iteration so the two multiply chains interleave.
template<class F>
__global__ void __launch_bounds__(kBlock)
    philox_fill_fast(PhiloxCall a, PhiloxLane lane, uint32_t x0, F f)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const F g = stage_table(f, smem);

    const uint32_t vec_n  = static_cast<uint32_t>(a.vec_n);
    const uint32_t stride = gridDim.x * kBlock;
    uint32_t       j      = blockIdx.x * kBlock + threadIdx.x;
    for(; j + stride < vec_n; j += 2 * stride)
    {
        const uint4 b0 = philox_block_lane(x0 + j, lane, a.keys);
        const uint4 b1 = philox_block_lane(x0 + j + stride, lane, a.keys);
        // both transforms before either store, so that their chains can interleave
        const uint4 v0 = philox_vec(g, b0);
        const uint4 v1 = philox_vec(g, b1);
        store16_cs(a.vec + static_cast<size_t>(j) * 16, v0);
        store16_cs(a.vec + static_cast<size_t>(j + stride) * 16, v1);
    }
    if(j < vec_n)
        store16_cs(a.vec + static_cast<size_t>(j) * 16, philox_vec(g, philox_block_lane(x0 + j, lane, a.keys)));

    if(blockIdx.x == 0 && threadIdx.x == 0)
    {
        using T = typename F::T;
        if(a.head > 0)
            philox_scalar_run(a, g, 0, reinterpret_cast<T*>(a.data), a.head);
        if(a.tail > 0)
            philox_scalar_run(a, g, 4 * a.vec_n + a.head, reinterpret_cast<T*>(a.data) + (a.n - a.tail),
                              a.tail);
    }
}

// The same output contract on the host (host generators without a GPU): every vector by
// the general rule of philox_fill, the head and tail by the same sequential run.
template<class F>
static rocrand_status philox_run_host(const PhiloxCall& a, const F& f)
{
    host_parallel_for(a.vec_n, [&](unsigned long long j0, unsigned long long j1) {
        for(unsigned long long j = j0; j < j1; j++)
        {
            const uint32_t           adj = (j & (kPhiloxRefStride - 1)) == 0 ? a.start0 : a.head;
            const unsigned long long q   = a.s0 + adj + 4 * j;
            const uint4              c   = ctr_add(a.c0, q >> 2);
            const uint32_t           s   = static_cast<uint32_t>(q & 3);
            uint4                    b   = philox_block(c, a.keys);
            if(s != 0)
                b = interleave4(b, philox_block(ctr_add(c, 1), a.keys), s);
            const uint4 v = philox_vec(f, b);
            std::memcpy(a.vec + j * 16, &v, 16);
        }
    });
    using T = typename F::T;
    if(a.head > 0)
        philox_scalar_run(a, f, 0, reinterpret_cast<T*>(a.data), a.head);
    if(a.tail > 0)
    {
        const unsigned long long pos = 4 * a.vec_n + ((a.vec_n % kPhiloxRefStride) == 0 ? a.start0 : a.head);
        philox_scalar_run(a, f, pos, reinterpret_cast<T*>(a.data) + (a.n - a.tail), a.tail);
    }
    return ROCRAND_STATUS_SUCCESS;
}

template<class F>
static rocrand_status launch_philox(PhiloxCall a, const F& f, cudaStream_t stream)
{
    const size_t smem    = table_smem_bytes(f);
    const bool   aligned = a.start0 == a.head && ((a.s0 + a.head) & 3u) == 0;
    const unsigned long long work = a.vec_n > 0 ? a.vec_n : 1;
    if(aligned)
    {
        const uint4 cbase = ctr_add(a.c0, (a.s0 + a.head) >> 2);
        // 32-bit indices in the fast kernel: keep j + 2*stride below 2^32 too.
        if(static_cast<unsigned long long>(cbase.x) + a.vec_n <= (1ull << 32)
           && a.vec_n < (1ull << 31))
        {
            const PhiloxLane lane = philox_lane(cbase, a.keys);
            auto             k    = philox_fill_fast<F>;
            k<<<grid_for(k, (work + 1) / 2, smem), kBlock, smem, stream>>>(a, lane, cbase.x, f);
            return launch_status();
        }
        auto k = philox_fill<F, true>;
        k<<<grid_for(k, work, smem), kBlock, smem, stream>>>(a, f);
    }
    else
    {
        auto k = philox_fill<F, false>;
        k<<<grid_for(k, work, smem), kBlock, smem, stream>>>(a, f);
    }
    return launch_status();
}

// ---------------------------------------------------------------------------------------

PhiloxGenerator::PhiloxGenerator() = default;
PhiloxGenerator::~PhiloxGenerator() = default;

// Output `index` of distribution d comes from stream value index * iw / ow (index a multiple
// of ow, output aligned to the distribution's vector), so the position is that offset.
rocrand_status PhiloxGenerator::set_output_position(Dist d, unsigned long long index)
{
    if(d == Dist::U64)
        return ROCRAND_STATUS_TYPE_ERROR;
    DistParams p;
    return with_functor(d, p, [&](auto f) -> rocrand_status {
        using F = decltype(f);
        if(index % F::ow != 0)
            return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
        return set_offset(index / F::ow * F::iw);
    });
}

rocrand_status PhiloxGenerator::init()
{
    if(m_initialized)
        return ROCRAND_STATUS_SUCCESS;
    // the Poisson tables are allocated here, as the reference's generators do in init(), so
    // that a generate call recorded by a stream capture allocates nothing
    const rocrand_status st = m_poisson.reserve();
    if(st != ROCRAND_STATUS_SUCCESS)
        return st;
    // seed(seed, subsequence 0, offset) (philox4x32_10.hpp:291-306, engine seed :134-141)
    m_pos = CounterPos{};
    m_pos.advance(m_offset);
    m_initialized = true;
    return ROCRAND_STATUS_SUCCESS;
}

rocrand_status PhiloxGenerator::set_order(rocrand_ordering order)
{
    // philox4x32_10.hpp:258-278: DEFAULT, DYNAMIC, BEST, LEGACY.  All give the same
    // output on this build.
    switch(order)
    {
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

rocrand_status PhiloxGenerator::generate(void* data, size_t n, Dist d, const DistParams& p)
{
    if(d == Dist::U64)
        return ROCRAND_STATUS_TYPE_ERROR; // 32-bit engine (philox4x32_10.hpp:359-375)
    rocrand_status st = init();
    if(st != ROCRAND_STATUS_SUCCESS)
        return st;
    if(data == nullptr)
        return ROCRAND_STATUS_SUCCESS;
    const size_t tsize = dist_elem_size(d);
    if(reinterpret_cast<uintptr_t>(data) % tsize != 0)
        return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE; // not even element-aligned

    st = with_functor(d, p, [&](auto f) -> rocrand_status {
        using F                    = decltype(f);
        constexpr unsigned iw      = F::iw;
        constexpr unsigned ow      = F::ow;
        constexpr unsigned fow     = (4 / iw) * ow; // elements per 16-byte vector
        const uintptr_t    addr    = reinterpret_cast<uintptr_t>(data);
        const size_t       mis     = (fow - addr / tsize % fow) % fow;
        PhiloxCall         a;
        a.keys   = philox_keys(m_seed);
        a.c0     = m_pos.counter;
        a.s0     = m_pos.sub;
        a.head   = static_cast<uint32_t>(n < mis ? n : mis);
        a.tail   = static_cast<uint32_t>((n - a.head) % fow);
        a.vec_n  = (n - a.head) / fow;
        a.start0 = a.head > 0 ? (a.head + ow - 1) / ow * iw : 0;
        a.n      = n;
        a.data   = static_cast<unsigned char*>(data);
        a.vec    = a.data + mis * tsize;
        if(n == 0)
            return ROCRAND_STATUS_SUCCESS;
        const rocrand_status s = m_host_exec ? philox_run_host(a, f) : launch_philox(a, f, m_stream);
        if(s == ROCRAND_STATUS_SUCCESS)
            m_pos.advance(static_cast<unsigned long long>((n + ow - 1) / ow) * iw);
        return s;
    });
    return st;
}

// Poisson values of a fresh Philox4x32-10 stream (seed, offset) with a caller-supplied
// table: used by the entry point that allocates nothing (noalloc.cu).
rocrand_status philox_poisson_with_table(unsigned long long seed, unsigned long long offset,
                                         unsigned int* data, size_t n, const DistParams& p,
                                         cudaStream_t stream)
{
    if(data == nullptr || n == 0)
        return ROCRAND_STATUS_SUCCESS;
    CounterPos pos;
    pos.advance(offset);
    const uintptr_t addr = reinterpret_cast<uintptr_t>(data);
    if(addr % sizeof(unsigned int) != 0)
        return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
    const size_t mis = (4 - addr / sizeof(unsigned int) % 4) % 4;
    PhiloxCall   a;
    a.keys   = philox_keys(seed);
    a.c0     = pos.counter;
    a.s0     = pos.sub;
    a.head   = static_cast<uint32_t>(n < mis ? n : mis);
    a.tail   = static_cast<uint32_t>((n - a.head) % 4);
    a.vec_n  = (n - a.head) / 4;
    a.start0 = a.head; // iw = ow = 1
    a.n      = n;
    a.data   = reinterpret_cast<unsigned char*>(data);
    a.vec    = a.data + mis * sizeof(unsigned int);
    if(p.huge)
        return launch_philox(a, FnPoissonHuge{p.sqrt_lambda, p.lambda}, stream);
    return launch_philox(a, FnPoisson{p.thr, p.alias, p.size, p.offset}, stream);
}

rocrand_status PhiloxGenerator::batch_descriptor(uint32_t dist, double p0, double p1, void* data,
                                                size_t n, BatchReq& r, cudaStream_t stream)
{
    rocrand_status st = init();
    if(st != ROCRAND_STATUS_SUCCESS)
        return st;
    r             = BatchReq{};
    r.kind        = BK_PHILOX;
    r.philox.keys = philox_keys(m_seed);
    r.philox.c0   = m_pos.counter;
    r.philox.s0   = m_pos.sub;
    st            = batch_set_dist(r, dist, p0, p1, stream);
    if(st == ROCRAND_STATUS_SUCCESS)
        st = batch_layout(r, data, n);
    if(st != ROCRAND_STATUS_SUCCESS)
        return st;
    unsigned iw, ow;
    batch_widths(BK_PHILOX, dist, iw, ow);
    m_pos.advance(static_cast<unsigned long long>((n + ow - 1) / ow) * iw);
    return ROCRAND_STATUS_SUCCESS;
}

rocrand_status PhiloxGenerator::generate_poisson(unsigned int* data, size_t n, double lambda)
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

} // namespace rb200
