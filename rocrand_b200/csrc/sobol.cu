// sobol.cu -- Sobol32, scrambled Sobol32, Sobol64 and scrambled Sobol64 quasi-random
// generators.
//
// Output contract of the reference (library/src/rng/sobol.hpp:72-256, 618-717): the output is
// dimension-major, out[d * N + i] = dist(x_d(offset + i)) with N = n / dims, where x_d(k) is
// the XOR of the direction vectors of dimension d selected by the bits of the Gray code
// k ^ (k >> 1) (rocrand_sobol32.h:122-170); the scrambled variants XOR the result with a
// per-dimension constant which, as the reference's generator is written (sobol.hpp:514),
// is word d of the scrambled direction-vector table.  The point counter is 32-bit and
// advances by N per call.
//
// B200 kernel: grid.y = dimension (its 32/64 vectors staged in shared memory), each thread
// produces a run of consecutive points by Gray-code steps (one XOR each) and leaps ahead by a
// power-of-two stride with two XORs (the leap-frog of rocrand_sobol32.h:140-159), writing
// 16-byte vectors where the row is aligned.  Distributions are applied in registers.
#include "common.hpp"
#include "dist.cuh"
#include "generators.hpp"
#include "launch.cuh"
#include "poisson.hpp"
#include "batch.hpp"
#include "sobol_dist.cuh"
#include "host_exec.hpp"
#include "sobol_tables.hpp"

#include <algorithm>
#include <type_traits>

namespace rb200
{

template<class W>
struct SobolCall
{
    const W*           vectors; // dims x B
    const W*           scramble; // scrambled table, read at flat index dim (nullptr: plain)
    unsigned char*     data;
    unsigned long long n;       // points per dimension
    unsigned long long chunk;   // points per block: a multiple of PPT * kBlock
    uint32_t           offset;
    SobolParams        p;
};

// Points per block for `dims` dimensions of n points each, blocks taking whole groups of
// `group` points, on a GPU holding `wave` resident blocks: among the block counts per
// dimension that fill k = 1 .. 64 waves (floor(k wave / dims) and one more), the one whose
// grid leaves the least of its last wave idle, the fewest blocks on ties.
inline unsigned long long sobol_chunk(unsigned long long n, unsigned long long dims, unsigned long long group,
                                      unsigned long long wave)
{
    if(wave == 0)
        wave = 1;
    const unsigned long long groups     = (n + group - 1) / group;
    unsigned long long       best_chunk = groups * group;
    unsigned long long       best_nb    = 1;
    double                   best_use   = 0.0;
    auto                     consider   = [&](unsigned long long b) {
        b                              = b < 1 ? 1 : (b > groups ? groups : b);
        const unsigned long long chunk = (groups + b - 1) / b * group;
        const unsigned long long nb    = (n + chunk - 1) / chunk;
        const unsigned long long waves = (nb * dims + wave - 1) / wave;
        const double             use   = static_cast<double>(nb * dims) / static_cast<double>(waves * wave);
        if(use > best_use + 1e-3 || (use > best_use - 1e-3 && nb < best_nb))
        {
            best_chunk = chunk;
            best_nb    = nb;
            best_use   = use > best_use ? use : best_use;
        }
    };
    for(unsigned long long k = 1; k <= 64; k++)
    {
        consider(k * wave / dims);
        consider(k * wave / dims + 1);
    }
    return best_chunk;
}

template<class W, SobolKind K>
__global__ void __launch_bounds__(kBlock) sobol_fill(SobolCall<W> a)
{
    using T                = typename SobolOut<K, W>::T;
    constexpr int      B   = 8 * sizeof(W);
    constexpr unsigned PPT = sizeof(T) >= 4 ? 4u : 16u / sizeof(T);
    // 64-bit index for Sobol64 (its engine counter is 64-bit), 32-bit for Sobol32.
    using I = W;

    __shared__ W v[B];
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t dim = blockIdx.y;
    if(threadIdx.x < B)
        v[threadIdx.x] = a.vectors[static_cast<size_t>(dim) * B + threadIdx.x];
    const double* cdf = nullptr;
    if constexpr(K == SobolKind::POISSON)
    {
        double* s = reinterpret_cast<double*>(smem);
        for(uint32_t k = threadIdx.x; k < a.p.size; k += blockDim.x)
            s[k] = a.p.cdf[k];
        cdf = s;
    }
    __syncthreads();

    const W            c      = a.scramble ? a.scramble[dim] : W(0);
    T*                 row    = reinterpret_cast<T*>(a.data) + static_cast<size_t>(dim) * a.n;
    // block x covers points [x chunk, (x + 1) chunk) of its dimension, its threads leap-frog
    // through them by the power-of-two stride PPT * kBlock
    constexpr unsigned long long stride = static_cast<unsigned long long>(PPT) * kBlock;
    constexpr uint32_t           lg     = PPT == 4 ? 10u : (PPT == 8 ? 11u : 12u); // log2(stride)
    static_assert((1ull << lg) == stride, "stride is a power of two");
    const unsigned long long begin = static_cast<unsigned long long>(blockIdx.x) * a.chunk;
    const unsigned long long end   = a.n < begin + a.chunk ? a.n : begin + a.chunk;
    unsigned long long       p     = begin + static_cast<unsigned long long>(threadIdx.x) * PPT;
    if(p >= end)
        return;
    const bool         vec_ok = (reinterpret_cast<uintptr_t>(row) % (PPT * sizeof(T))) == 0;

    // The engine starts at the 32-bit sum offset + p (sobol.hpp:191-196) and then counts in
    // its own width.
    I i = static_cast<I>(static_cast<uint32_t>(a.offset + static_cast<uint32_t>(p)));
    W x = 0;
    {
        const I g = i ^ (i >> 1);
#pragma unroll
        for(int b = 0; b < B; b++)
            if((g >> b) & 1)
                x ^= v[b];
    }
    for(; p < end; p += stride)
    {
        T out[PPT];
        W xx = x;
        I ii = i;
#pragma unroll
        for(unsigned k = 0; k < PPT; k++)
        {
            out[k] = sobol_apply<K, W>(xx ^ c, a.p, cdf);
            xx ^= v[rzb(ii)];
            ii++;
        }
        if(vec_ok && p + PPT <= a.n)
        {
            constexpr unsigned VB = PPT * sizeof(T);
            if constexpr(VB == 16)
            {
                uint4 w;
                memcpy(&w, out, 16);
                __stcs(reinterpret_cast<uint4*>(row + p), w);
            }
            else
            {
                static_assert(VB == 32, "vector");
                uint4 w[2];
                memcpy(w, out, 32);
                __stcs(reinterpret_cast<uint4*>(row + p), w[0]);
                __stcs(reinterpret_cast<uint4*>(row + p) + 1, w[1]);
            }
        }
        else
        {
            for(unsigned k = 0; k < PPT && p + k < a.n; k++)
                row[p + k] = out[k];
        }
        // leap-frog by the power-of-two stride 2^lg: Gray-code bit lg-1 flips, and the bit of
        // the lowest zero of i above the low lg bits (rocrand_sobol32.h:140-159)
        x ^= v[lg - 1];
        x ^= v[rzb(static_cast<I>(i | static_cast<I>(stride - 1)))];
        i += static_cast<I>(stride);
    }
}

// ---------------------------------------------------------------------------------------

template<bool kIs64, bool kScrambled>
class SobolGenerator final : public rocrand_generator_base_type
{
    using W = std::conditional_t<kIs64, unsigned long long, uint32_t>;

public:
    bool set_host_execution() override
    {
        m_host_exec = true;
        m_poisson.set_host();
        return true;
    }
    rocrand_rng_type type() const override
    {
        if(kIs64)
            return kScrambled ? ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL64 : ROCRAND_RNG_QUASI_SOBOL64;
        return kScrambled ? ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL32 : ROCRAND_RNG_QUASI_SOBOL32;
    }
    rocrand_status init() override
    {
        if(!m_initialized)
        {
            // the Poisson tables are allocated here, as the reference's generators do in init(), so
            // that a generate call recorded by a stream capture allocates nothing
            const rocrand_status st = m_poisson.reserve();
            if(st != ROCRAND_STATUS_SUCCESS)
                return st;
            // likewise the device tables every generate call reads (uploaded once per device)
            lr::Table lt;
            if(!m_host_exec
               && (sobol_device_vectors(kIs64, kScrambled) == nullptr || !logf_replay_device(lt)))
                return ROCRAND_STATUS_ALLOCATION_FAILED;
            m_current     = static_cast<uint32_t>(m_offset); // 32-bit counter (sobol.hpp:604)
            m_initialized = true;
        }
        return ROCRAND_STATUS_SUCCESS;
    }
    rocrand_status set_seed(unsigned long long) override { return ROCRAND_STATUS_SUCCESS; }
    rocrand_status set_offset(unsigned long long offset) override
    {
        m_offset      = offset;
        m_initialized = false;
        return ROCRAND_STATUS_SUCCESS;
    }
    rocrand_status set_order(rocrand_ordering order) override
    {
        if(order != ROCRAND_ORDERING_QUASI_DEFAULT)
            return ROCRAND_STATUS_OUT_OF_RANGE;
        m_initialized = false;
        return ROCRAND_STATUS_SUCCESS;
    }
    rocrand_status set_dimensions(unsigned int dims) override
    {
        if(dims < 1 || dims > kSobolDims)
            return ROCRAND_STATUS_OUT_OF_RANGE;
        m_dims        = dims;
        m_initialized = false;
        return ROCRAND_STATUS_SUCCESS;
    }

    rocrand_status batch_descriptor(uint32_t dist, double p0, double p1, void* data, size_t n,
                                    BatchReq& r, cudaStream_t stream) override
    {
        if(kIs64 || kScrambled || m_dims != 1)
            return ROCRAND_STATUS_TYPE_ERROR;
        rocrand_status st = init();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        r              = BatchReq{};
        r.kind         = BK_SOBOL32;
        r.sobol_offset = m_current;
        r.sobol_v      = static_cast<const uint32_t*>(sobol_device_vectors(false, false));
        if(r.sobol_v == nullptr)
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        st = batch_set_dist(r, dist, p0, p1, stream);
        if(st == ROCRAND_STATUS_SUCCESS)
            st = batch_layout(r, data, n);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        m_current += static_cast<uint32_t>(n);
        return ROCRAND_STATUS_SUCCESS;
    }

    rocrand_status generate(void* data, size_t n, Dist d, const DistParams& dp) override
    {
        if(!kIs64 && d == Dist::U64)
            return ROCRAND_STATUS_TYPE_ERROR;
        if(n % m_dims != 0)
            return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
        rocrand_status st = init();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        if(data == nullptr)
            return ROCRAND_STATUS_SUCCESS;
        if(reinterpret_cast<uintptr_t>(data) % dist_elem_size(d) != 0)
            return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
        SobolParams p{};
        p.mean_f = dp.mean_f;
        p.std_f  = dp.std_f;
        p.mean_d = dp.mean_d;
        p.std_d  = dp.std_d;
        if(d == Dist::NORMAL_F16 || d == Dist::LOGNORMAL_F16)
        {
            p.mean_f = __half2float(__ushort_as_half(dp.mean_h));
            p.std_f  = __half2float(__ushort_as_half(dp.std_h));
        }
        p.cdf         = dp.cdf;
        p.size        = dp.size;
        p.offset      = dp.offset;
        p.lambda      = dp.lambda;
        p.sqrt_lambda = dp.sqrt_lambda;
        if(!m_host_exec
           && (d == Dist::NORMAL_F32 || d == Dist::LOGNORMAL_F32 || d == Dist::NORMAL_F16
               || d == Dist::LOGNORMAL_F16)
           && !logf_replay_device(p.logf))
            return ROCRAND_STATUS_INTERNAL_ERROR;
        switch(d)
        {
            case Dist::U32: st = launch<SobolKind::UINT>(data, n, p); break;
            case Dist::U64: st = launch<SobolKind::ULL>(data, n, p); break;
            case Dist::U8: st = launch<SobolKind::UCHAR>(data, n, p); break;
            case Dist::U16: st = launch<SobolKind::USHORT>(data, n, p); break;
            case Dist::F32: st = launch<SobolKind::FLOAT>(data, n, p); break;
            case Dist::F64: st = launch<SobolKind::DOUBLE>(data, n, p); break;
            case Dist::F16: st = launch<SobolKind::HALF>(data, n, p); break;
            case Dist::NORMAL_F32: st = launch<SobolKind::NORMAL_F>(data, n, p); break;
            case Dist::NORMAL_F64: st = launch<SobolKind::NORMAL_D>(data, n, p); break;
            case Dist::NORMAL_F16: st = launch<SobolKind::NORMAL_H>(data, n, p); break;
            case Dist::LOGNORMAL_F32: st = launch<SobolKind::LOGNORMAL_F>(data, n, p); break;
            case Dist::LOGNORMAL_F64: st = launch<SobolKind::LOGNORMAL_D>(data, n, p); break;
            case Dist::LOGNORMAL_F16: st = launch<SobolKind::LOGNORMAL_H>(data, n, p); break;
            case Dist::POISSON:
                st = dp.huge ? launch<SobolKind::POISSON_HUGE>(data, n, p)
                             : launch<SobolKind::POISSON>(data, n, p);
                break;
            default: return ROCRAND_STATUS_TYPE_ERROR;
        }
        if(st == ROCRAND_STATUS_SUCCESS)
            m_current += static_cast<uint32_t>(n / m_dims);
        return st;
    }

    rocrand_status generate_poisson(unsigned int* data, size_t n, double lambda) override
    {
        DistParams p;
        // The quasi-random generators use the CDF form of the table (sobol.hpp:498-499).
        const rocrand_status st = m_poisson.get(lambda, m_stream, true, p);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        return generate(data, n, Dist::POISSON, p);
    }

private:
    template<SobolKind K>
    rocrand_status launch(void* data, size_t n, const SobolParams& p)
    {
        using T                = typename SobolOut<K, W>::T;
        constexpr unsigned PPT = sizeof(T) >= 4 ? 4u : 16u / sizeof(T);
        if(m_host_exec)
            return run_host<K>(data, n, p);
        const W*           vec = static_cast<const W*>(sobol_device_vectors(kIs64, kScrambled));
        if(vec == nullptr)
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        const unsigned long long N = n / m_dims;
        if(N == 0)
            return ROCRAND_STATUS_SUCCESS;
        SobolCall<W> a;
        a.vectors  = vec;
        a.scramble = kScrambled ? vec : nullptr;
        a.data     = static_cast<unsigned char*>(data);
        a.n        = N;
        a.offset   = m_current;
        a.p        = p;
        // blocks per dimension: whole groups of PPT * kBlock points each, as many as fill the
        // GPU's resident blocks in nearly whole waves
        const size_t             smem  = K == SobolKind::POISSON ? p.size * sizeof(double) : 0;
        constexpr unsigned long long group = static_cast<unsigned long long>(PPT) * kBlock;
        const void* const kernel = reinterpret_cast<const void*>(sobol_fill<W, K>);
        if(m_chunk_kernel != kernel || m_chunk_n != N || m_chunk_smem != smem || m_chunk_dims != m_dims)
        {
            const unsigned long long wave
                = static_cast<unsigned long long>(device_info().sm_count) * blocks_per_sm(kernel, smem);
            m_chunk        = sobol_chunk(N, m_dims, group, wave);
            m_chunk_kernel = kernel;
            m_chunk_n      = N;
            m_chunk_smem   = smem;
            m_chunk_dims   = m_dims;
        }
        a.chunk                        = m_chunk;
        const unsigned long long nb    = (N + a.chunk - 1) / a.chunk;
        sobol_fill<W, K><<<dim3(static_cast<unsigned>(nb), m_dims), kBlock, smem, m_stream>>>(a);
        return launch_status();
    }

    // The same output on the host (host generators without a GPU): point i of dimension d is
    // the XOR of d's direction vectors over the set bits of Gray(i), with i counted from the
    // 32-bit start as the kernel counts it, and the distribution applied to it.
    template<SobolKind K>
    rocrand_status run_host(void* data, size_t n, const SobolParams& p)
    {
        using T                     = typename SobolOut<K, W>::T;
        using I                     = W;
        constexpr int         B     = 8 * sizeof(W);
        const SobolTables&    t     = sobol_tables();
        if(!t.ok)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        const W* const vec = reinterpret_cast<const W*>(
            kIs64 ? static_cast<const void*>(kScrambled ? t.sv64.data() : t.v64.data())
                  : static_cast<const void*>(kScrambled ? t.sv32.data() : t.v32.data()));
        const unsigned long long N = n / m_dims;
        const uint32_t           offset = m_current;
        host_parallel_for(static_cast<unsigned long long>(m_dims) * N,
                          [&](unsigned long long b0, unsigned long long b1) {
            while(b0 < b1)
            {
                const unsigned long long dim = b0 / N, p0 = b0 % N;
                const unsigned long long p1  = std::min<unsigned long long>(N, p0 + (b1 - b0));
                const W* const v   = vec + dim * B;
                const W        c   = kScrambled ? vec[dim] : W(0);
                T* const       row = static_cast<T*>(data) + dim * N;
                I              i   = static_cast<I>(static_cast<uint32_t>(offset + static_cast<uint32_t>(p0)));
                W              x   = 0;
                const I        g   = i ^ (i >> 1);
                for(int bit = 0; bit < B; bit++)
                    if((g >> bit) & 1)
                        x ^= v[bit];
                for(unsigned long long q = p0; q < p1; q++)
                {
                    row[q] = sobol_apply<K, W>(x ^ c, p, p.cdf);
                    x ^= v[rzb(i)];
                    i++;
                }
                b0 += p1 - p0;
            }
        });
        return ROCRAND_STATUS_SUCCESS;
    }

    unsigned long long m_offset      = 0;
    uint32_t           m_current     = 0;
    unsigned int       m_dims        = 1;
    bool               m_initialized = false;
    PoissonCache       m_poisson;
    // the block size in points of the last launch shape (kernel, points per dimension,
    // shared memory, dimensions), chosen once per shape
    const void*        m_chunk_kernel = nullptr;
    unsigned long long m_chunk_n      = 0;
    size_t             m_chunk_smem   = 0;
    unsigned int       m_chunk_dims   = 0;
    unsigned long long m_chunk        = 0;
};

rocrand_generator_base_type* make_sobol(rocrand_rng_type t)
{
    switch(t)
    {
        case ROCRAND_RNG_QUASI_DEFAULT:
        case ROCRAND_RNG_QUASI_SOBOL32: return new SobolGenerator<false, false>();
        case ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL32: return new SobolGenerator<false, true>();
        case ROCRAND_RNG_QUASI_SOBOL64: return new SobolGenerator<true, false>();
        case ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL64: return new SobolGenerator<true, true>();
        default: return nullptr;
    }
}

} // namespace rb200
