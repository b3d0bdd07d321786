// mtgp32.cu -- MTGP32: 512 block generators, each its own published recurrence.
//
// Output contract (library/src/rng/mtgp32.hpp:232-305, rocrand_mtgp32.h): generator b
// (one of 512, config/config_defaults.hpp:48-52) belongs to block b of 256 threads.  One
// block step advances the generator by 256 values: thread t computes
//   r = para_rec(s[k+t], s[k+t+1], s[k+t+pos]),  s[k+t+351] = r,  out = temper(r, s[k+t+pos-1])
// on a 1024-word state ring (k = the ring offset, then k += 256).  Output vector j is thread
// j % 256 of generator (j / 256) % 512 in round j / 131072; a distribution call takes its iw
// inputs from iw successive steps.  After the full rounds every generator steps once more
// when the last round is partial (writing only the vectors that exist), and once more when
// the call has a head or tail, which the threads at vector indices vec_n_up and
// vec_n_up + 1 write.  State and offset carry over to the next call.
//
// B200 layout: the rings and offsets of the 512 generators live in HBM (2 MiB); each block
// keeps its ring in shared memory for the whole call (one __syncthreads per step: a step's
// reads stop 1 short of its first write, the next step reads what it wrote), its parameter
// set in registers and shared memory.  The parameter sets are the published MTGP32 11213
// dynamic-creator sets (rocrand_b200/data/mtgp32_params.bin, embedded by mtgp32_data.S).
#include "common.hpp"
#include "dist.cuh"
#include "generators.hpp"
#include "host_exec.hpp"
#include "launch.cuh"
#include "stateful_engines.cuh"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

extern "C" const unsigned char rb200_mtgp32_params_begin[];
extern "C" const unsigned char rb200_mtgp32_params_end[];

namespace rb200
{
namespace
{

constexpr int      kMtgpN     = 351;
constexpr int      kMtgpState = 1024;
constexpr int      kMtgpMask  = 1023;
constexpr uint32_t kMtgpGens  = 512;
constexpr uint32_t kMtgpBlock = 256;
constexpr int      kMtgpWords = 36; // pos, sh1, sh2, tbl[16], tmp_tbl[16], mask

struct MtgpArgs
{
    uint32_t*          rings;   // [512][1024]
    int*               offsets; // [512]
    const uint32_t*    params;  // [512][36]
    unsigned char*     data;
    unsigned char*     vec;
    unsigned long long n, vec_n, vec_n_down, vec_n_up;
    uint32_t           head, tail;
};

// Units a thread transforms side by side in the main loop: four fp64 Box-Muller chains,
// two fp32 ones.
template<class F>
constexpr unsigned kMtgpUnits
    = (std::is_same<F, FnNormalD>::value || std::is_same<F, FnLogNormalD>::value) ? 4u : 2u;

// 4 blocks of 256 threads per SM (at most 64 registers): all 512 block generators resident
// at once on 148 SMs.
template<class F>
__global__ void __launch_bounds__(kMtgpBlock, 4) mtgp_fill(MtgpArgs a, F fw)
{
    __shared__ uint32_t        s[kMtgpState];
    __shared__ uint32_t        tbl[16], tmp[16];
    extern __shared__ unsigned char smem[];
    const F                    f = stage_table(fw, smem);
    const uint32_t             b = blockIdx.x, t = threadIdx.x;
    const uint32_t*            p = a.params + b * kMtgpWords;
    for(int i = t; i < kMtgpState; i += kMtgpBlock)
        s[i] = a.rings[b * kMtgpState + i];
    if(t < 16)
    {
        tbl[t] = p[3 + t];
        tmp[t] = p[19 + t];
    }
    const int      pos = static_cast<int>(p[0]);
    const uint32_t sh1 = p[1], sh2 = p[2], mask = p[35];
    int            k   = a.offsets[b];
    __syncthreads();

    // one block step: this thread's value, then every thread's writes become visible
    auto step = [&]() -> uint32_t {
        uint32_t x = (s[(k + t) & kMtgpMask] & mask) ^ s[(k + t + 1) & kMtgpMask];
        uint32_t y = s[(k + t + pos) & kMtgpMask];
        x ^= x << sh1;
        y                                 = x ^ (y >> sh2);
        const uint32_t r                  = y ^ tbl[y & 0x0f];
        s[(k + t + kMtgpN) & kMtgpMask]   = r;
        uint32_t tt                       = s[(k + t + pos - 1) & kMtgpMask];
        tt ^= tt >> 16;
        tt ^= tt >> 8;
        __syncthreads();
        k = (k + kMtgpBlock) & kMtgpMask;
        return r ^ tmp[tt & 0x0f];
    };

    using T                      = typename F::T;
    constexpr unsigned ow        = F::ow;
    constexpr unsigned VB        = ow * sizeof(T);
    const unsigned long long str = static_cast<unsigned long long>(kMtgpGens) * kMtgpBlock;
    unsigned long long index     = static_cast<unsigned long long>(b) * kMtgpBlock + t;
    uint32_t           in[F::iw];
    T                  out[ow];
    auto               gen = [&]() {
#pragma unroll
        for(unsigned i = 0; i < F::iw; i++)
            in[i] = step();
        f(in, out);
    };
    // index < vec_n_down and index < vec_n_up are the same in the whole block (both are
    // multiples of 256), so every thread takes every step
    if constexpr(long_transform<F>::value)
    {
        // U rounds' steps, then their transforms with no branch between them: the U
        // Box-Muller chains interleave instead of each waiting out its own latency
        constexpr unsigned U = kMtgpUnits<F>;
        while(index + (U - 1) * str < a.vec_n_down)
        {
            uint32_t in[U][F::iw];
#pragma unroll
            for(unsigned u = 0; u < U; u++)
#pragma unroll
                for(unsigned i = 0; i < F::iw; i++)
                    in[u][i] = step();
            T o[U][ow];
#pragma unroll
            for(unsigned u = 0; u < U; u++)
                f(in[u], o[u]);
#pragma unroll
            for(unsigned u = 0; u < U; u++)
                store_small(a.vec + (index + u * str) * VB, o[u]);
            index += U * str;
        }
    }
    while(index < a.vec_n_down)
    {
        gen();
        store_small(a.vec + index * VB, out);
        index += str;
    }
    if(index < a.vec_n_up)
    {
        gen();
        if(index < a.vec_n)
            store_small(a.vec + index * VB, out);
        index += str;
    }
    if(ow > 1 && (a.head > 0 || a.tail > 0))
    {
        gen();
        T* data = reinterpret_cast<T*>(a.data);
        if(index == a.vec_n_up)
            for(unsigned o = 0; o < a.head; o++)
                data[o] = out[o];
        if(index == a.vec_n_up + 1)
            for(unsigned o = 0; o < a.tail; o++)
                data[a.n - a.tail + o] = out[o];
    }
    for(int i = t; i < kMtgpState; i += kMtgpBlock)
        a.rings[b * kMtgpState + i] = s[i];
    if(t == 0)
        a.offsets[b] = k;
}

// mtgp_fill on the host (CPU path of the host generators): generator b's 256 threads take
// each block step in thread order -- a step's reads end before its first written word, so
// the order within a step does not change a value -- then every thread applies the
// distribution to its inputs and writes by mtgp_fill's rules.  Generators are independent.
template<class F>
void mtgp_fill_host(const MtgpArgs& a, const F& f)
{
    using T                      = typename F::T;
    constexpr unsigned iw        = F::iw;
    constexpr unsigned ow        = F::ow;
    constexpr unsigned VB        = ow * sizeof(T);
    const unsigned long long str = static_cast<unsigned long long>(kMtgpGens) * kMtgpBlock;
    host_parallel_for(
        kMtgpGens,
        [&](unsigned long long b0, unsigned long long b1) {
            std::vector<uint32_t> vals(static_cast<size_t>(iw) * kMtgpBlock);
            std::vector<T>        outs(static_cast<size_t>(ow) * kMtgpBlock);
            for(unsigned long long b = b0; b < b1; b++)
            {
                uint32_t*       s    = a.rings + b * kMtgpState;
                const uint32_t* p    = a.params + b * kMtgpWords;
                const int       pos  = static_cast<int>(p[0]);
                const uint32_t  sh1 = p[1], sh2 = p[2], mask = p[35];
                const uint32_t* tbl  = p + 3;
                const uint32_t* tmp  = p + 19;
                int             k    = a.offsets[b];
                // iw block steps, then the distribution on each thread's inputs
                auto gen = [&]() {
                    for(unsigned i = 0; i < iw; i++)
                    {
                        for(uint32_t t = 0; t < kMtgpBlock; t++)
                        {
                            uint32_t x = (s[(k + t) & kMtgpMask] & mask) ^ s[(k + t + 1) & kMtgpMask];
                            uint32_t y = s[(k + t + pos) & kMtgpMask];
                            x ^= x << sh1;
                            y                               = x ^ (y >> sh2);
                            const uint32_t r                = y ^ tbl[y & 0x0f];
                            s[(k + t + kMtgpN) & kMtgpMask] = r;
                            uint32_t tt                     = s[(k + t + pos - 1) & kMtgpMask];
                            tt ^= tt >> 16;
                            tt ^= tt >> 8;
                            vals[t * iw + i] = r ^ tmp[tt & 0x0f];
                        }
                        k = (k + kMtgpBlock) & kMtgpMask;
                    }
                    for(uint32_t t = 0; t < kMtgpBlock; t++)
                        f(&vals[t * iw], &outs[t * ow]);
                };
                unsigned long long index = b * kMtgpBlock; // thread 0's vector index
                while(index < a.vec_n_down)
                {
                    gen();
                    std::memcpy(a.vec + index * VB, outs.data(), VB * kMtgpBlock);
                    index += str;
                }
                if(index < a.vec_n_up)
                {
                    gen();
                    for(uint32_t t = 0; t < kMtgpBlock; t++)
                        if(index + t < a.vec_n)
                            std::memcpy(a.vec + (index + t) * VB, &outs[t * ow], VB);
                    index += str;
                }
                if(ow > 1 && (a.head > 0 || a.tail > 0))
                {
                    gen();
                    T* data = reinterpret_cast<T*>(a.data);
                    for(uint32_t t = 0; t < kMtgpBlock; t++)
                    {
                        if(index + t == a.vec_n_up)
                            for(unsigned o = 0; o < a.head; o++)
                                data[o] = outs[t * ow + o];
                        if(index + t == a.vec_n_up + 1)
                            for(unsigned o = 0; o < a.tail; o++)
                                data[a.n - a.tail + o] = outs[t * ow + o];
                    }
                }
                a.offsets[b] = k;
            }
        },
        2);
}

// Parameter sets on each device, uploaded once.
const uint32_t* device_params()
{
    static std::mutex                   mu;
    static std::vector<const uint32_t*> ptr(64, nullptr);
    const int                           dev = device_info().device;
    std::lock_guard<std::mutex>         lock(mu);
    if(ptr[dev])
        return ptr[dev];
    const size_t bytes = static_cast<size_t>(rb200_mtgp32_params_end - rb200_mtgp32_params_begin);
    const size_t want  = 12 + sizeof(uint32_t) * kMtgpWords * kMtgpGens;
    if(bytes != want || std::memcmp(rb200_mtgp32_params_begin, "RBMTGP01", 8) != 0)
        return nullptr;
    void* d = nullptr;
    if(cudaMalloc(&d, want - 12) != cudaSuccess)
        return nullptr;
    if(cudaMemcpy(d, rb200_mtgp32_params_begin + 12, want - 12, cudaMemcpyHostToDevice) != cudaSuccess)
    {
        cudaFree(d);
        return nullptr;
    }
    ptr[dev] = static_cast<const uint32_t*>(d);
    return ptr[dev];
}

class Mtgp32Generator final : public PseudoGeneratorBase
{
public:
    ~Mtgp32Generator() override
    {
        if(m_rings != nullptr)
            cudaFree(m_rings);
    }

    bool set_host_execution() override { return enable_host(); }

    rocrand_rng_type type() const override { return ROCRAND_RNG_PSEUDO_MTGP32; }

    // mtgp32.hpp:389-393: MTGP32 has no offset
    rocrand_status set_offset(unsigned long long offset) override
    {
        (void)offset;
        return ROCRAND_STATUS_TYPE_ERROR;
    }

    // mtgp32.hpp:395-416 (device generator: DYNAMIC accepted)
    rocrand_status set_order(rocrand_ordering order) override
    {
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

    rocrand_status init() override
    {
        if(m_initialized)
            return ROCRAND_STATUS_SUCCESS;
        // the Poisson tables are allocated here, as the reference's generators do in init(), so
        // that a generate call recorded by a stream capture allocates nothing
        if(m_poisson.reserve() != ROCRAND_STATUS_SUCCESS)
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        const size_t pbytes = static_cast<size_t>(rb200_mtgp32_params_end - rb200_mtgp32_params_begin);
        if(pbytes != 12 + sizeof(uint32_t) * kMtgpWords * kMtgpGens
           || std::memcmp(rb200_mtgp32_params_begin, "RBMTGP01", 8) != 0)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        m_params = m_host_exec ? reinterpret_cast<const uint32_t*>(rb200_mtgp32_params_begin + 12)
                               : device_params();
        if(m_params == nullptr)
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        constexpr size_t kRingWords = static_cast<size_t>(kMtgpGens) * kMtgpState;
        if(m_rings == nullptr && !m_host_exec)
        {
            if(cudaMalloc(&m_rings, sizeof(uint32_t) * kRingWords + sizeof(int) * kMtgpGens)
               != cudaSuccess)
            {
                m_rings = nullptr;
                return ROCRAND_STATUS_ALLOCATION_FAILED;
            }
        }
        // rocrand_make_state_mtgp32 / rocrand_mtgp32_init_state on the host (2 MiB)
        const auto*              host_params = reinterpret_cast<const uint32_t*>(rb200_mtgp32_params_begin + 12);
        std::vector<uint32_t>    rings(kRingWords, 0u);
        const unsigned long long seed = m_seed ^ (m_seed >> 32);
        for(uint32_t i = 0; i < kMtgpGens; i++)
        {
            const uint32_t* tbl    = host_params + i * kMtgpWords + 3;
            const uint32_t  hidden = tbl[4] ^ (tbl[8] << 16);
            uint32_t        tmp    = hidden;
            tmp += tmp >> 16;
            tmp += tmp >> 8;
            uint32_t* s = rings.data() + static_cast<size_t>(i) * kMtgpState;
            for(int k = 0; k < kMtgpN; k++)
                s[k] = (tmp & 0xffu) * 0x01010101u;
            s[0] = static_cast<uint32_t>(seed) + i + 1u;
            s[1] = hidden;
            for(uint32_t k = 1; k < static_cast<uint32_t>(kMtgpN); k++)
                s[k] ^= 1812433253u * (s[k - 1] ^ (s[k - 1] >> 30)) + k;
        }
        if(m_host_exec)
        {
            // the host copy: rings, then the 512 ring offsets
            m_hrings.assign(kRingWords + kMtgpGens, 0u);
            std::memcpy(m_hrings.data(), rings.data(), sizeof(uint32_t) * kRingWords);
            m_initialized = true;
            return ROCRAND_STATUS_SUCCESS;
        }
        // pageable sources: the copies have read them when cudaMemcpyAsync returns
        if(cudaMemcpyAsync(m_rings, rings.data(), sizeof(uint32_t) * kRingWords,
                           cudaMemcpyHostToDevice, m_stream)
               != cudaSuccess
           || cudaMemsetAsync(m_rings + kRingWords, 0, sizeof(int) * kMtgpGens, m_stream)
                  != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        m_initialized = true;
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
        constexpr unsigned ow   = F::ow;
        const uintptr_t    addr = reinterpret_cast<uintptr_t>(data);
        const size_t       mis  = (ow - addr / tsize % ow) % ow;
        MtgpArgs           a;
        uint32_t*          rings = m_host_exec ? m_hrings.data() : m_rings;
        a.rings      = rings;
        a.offsets    = reinterpret_cast<int*>(rings + static_cast<size_t>(kMtgpGens) * kMtgpState);
        a.params     = m_params;
        a.head       = static_cast<uint32_t>(n < mis ? n : mis);
        a.tail       = static_cast<uint32_t>((n - a.head) % ow);
        a.vec_n      = (n - a.head) / ow;
        a.n          = n;
        a.data       = static_cast<unsigned char*>(data);
        a.vec        = a.data + mis * tsize;
        const unsigned long long rem = a.vec_n % kMtgpBlock;
        a.vec_n_down = a.vec_n - rem;
        a.vec_n_up   = rem == 0 ? a.vec_n_down : a.vec_n_down + kMtgpBlock;
        // every call steps every generator (mtgp32.hpp:268-305), even with nothing to write
        if(m_host_exec)
        {
            mtgp_fill_host(a, f);
            return ROCRAND_STATUS_SUCCESS;
        }
        const size_t smem = table_smem_bytes(f);
        mtgp_fill<F><<<kMtgpGens, kMtgpBlock, smem, m_stream>>>(a, f);
        return launch_status();
    }

    uint32_t*       m_rings  = nullptr;
    const uint32_t* m_params = nullptr;
    // rings and offsets of the CPU path (the device layout, in host memory)
    std::vector<uint32_t> m_hrings;
};

} // namespace

rocrand_generator_base_type* make_mtgp32()
{
    return new Mtgp32Generator();
}

} // namespace rb200
