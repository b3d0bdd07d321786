// harness.cu -- test kernels of the device API (rocrand/rocrand_kernel.h).
//
// The same source is compiled twice: against this library's include/ (tests/devapi/
// Makefile, libdevapi_b200.so) and against the reference's own headers
// (oracle/Makefile.ref, oracle/_ref/libdevapi_ref.so), with the same nvcc flags; the GPU
// tests run both on the same inputs and compare the bytes.  TEST INFRASTRUCTURE ONLY.
//
// devapi_run: `threads` threads, thread t initialises one state of `engine` (seed, t, 7 t for
// the pseudo-random engines; direction vectors `vec`, scramble constant `scramble`, offset
// 5 t for Sobol) and makes `calls` calls of function `func`, each result stored in its own
// 32-byte slot: out[(t * calls + c) * 32].  A function an engine does not have stores
// nothing and the call returns 1; a launch error returns 2.
#include <rocrand/rocrand_kernel.h>
#include <rocrand/rocrand_mtgp32_11213.h>

#include <cuda_runtime.h>

#include <type_traits>
#include <utility>

namespace
{

#define DETECT(name, expr)                                                            \
    template<class S, class = void>                                                   \
    struct name : std::false_type                                                     \
    {};                                                                               \
    template<class S>                                                                 \
    struct name<S, std::void_t<decltype(expr)>> : std::true_type                      \
    {};

DETECT(has_rocrand2, rocrand2(std::declval<S*>()))
DETECT(has_rocrand4, rocrand4(std::declval<S*>()))
DETECT(has_uniform2, rocrand_uniform2(std::declval<S*>()))
DETECT(has_uniform4, rocrand_uniform4(std::declval<S*>()))
DETECT(has_uniform_double2, rocrand_uniform_double2(std::declval<S*>()))
DETECT(has_uniform_double4, rocrand_uniform_double4(std::declval<S*>()))
DETECT(has_normal2, rocrand_normal2(std::declval<S*>()))
DETECT(has_normal4, rocrand_normal4(std::declval<S*>()))
DETECT(has_normal_double2, rocrand_normal_double2(std::declval<S*>()))
DETECT(has_normal_double4, rocrand_normal_double4(std::declval<S*>()))
DETECT(has_log_normal2, rocrand_log_normal2(std::declval<S*>(), 0.0f, 1.0f))
DETECT(has_log_normal4, rocrand_log_normal4(std::declval<S*>(), 0.0f, 1.0f))
DETECT(has_log_normal_double2, rocrand_log_normal_double2(std::declval<S*>(), 0.0, 1.0))
DETECT(has_log_normal_double4, rocrand_log_normal_double4(std::declval<S*>(), 0.0, 1.0))
DETECT(has_poisson4, rocrand_poisson4(std::declval<S*>(), 1.0))
DETECT(has_discrete4, rocrand_discrete4(std::declval<S*>(), rocrand_discrete_distribution{}))
DETECT(has_skip, skipahead(1ull, std::declval<S*>()))
DETECT(has_skip_subsequence, skipahead_subsequence(1ull, std::declval<S*>()))
DETECT(has_skip_sequence, skipahead_sequence(1ull, std::declval<S*>()))

template<class T>
__device__ void put(unsigned char* slot, const T& v)
{
    static_assert(sizeof(T) <= 32, "slot");
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    for(unsigned i = 0; i < sizeof(T); i++)
        slot[i] = p[i];
}

struct Args
{
    int                                 func, calls;
    double                              p0, p1;
    unsigned long long                  seed;
    const void*                         vec;
    unsigned long long                  scramble;
    const rocrand_discrete_distribution_st* dist;
    unsigned char*                      out;
};

// one call of function f on state s into slot; false where the engine has no such function
template<class S>
__device__ bool call(S* s, int f, int c, const Args& a, unsigned char* slot)
{
    const float  mf = static_cast<float>(a.p0), sf = static_cast<float>(a.p1);
    const double md = a.p0, sd = a.p1;
    rocrand_discrete_distribution dd = const_cast<rocrand_discrete_distribution>(a.dist);
    switch(f)
    {
        case 0: put(slot, rocrand(s)); return true;
        case 1:
            if constexpr(has_rocrand4<S>::value)
            {
                put(slot, rocrand4(s));
                return true;
            }
            else if constexpr(has_rocrand2<S>::value)
            {
                put(slot, rocrand2(s));
                return true;
            }
            return false;
        case 2: put(slot, rocrand_uniform(s)); return true;
        case 3:
            if constexpr(has_uniform2<S>::value)
            {
                put(slot, rocrand_uniform2(s));
                return true;
            }
            return false;
        case 4:
            if constexpr(has_uniform4<S>::value)
            {
                put(slot, rocrand_uniform4(s));
                return true;
            }
            return false;
        case 5: put(slot, rocrand_uniform_double(s)); return true;
        case 6:
            if constexpr(has_uniform_double2<S>::value)
            {
                put(slot, rocrand_uniform_double2(s));
                return true;
            }
            return false;
        case 7:
            if constexpr(has_uniform_double4<S>::value)
            {
                put(slot, rocrand_uniform_double4(s));
                return true;
            }
            return false;
        case 8: put(slot, rocrand_normal(s)); return true;
        case 9:
            if constexpr(has_normal2<S>::value)
            {
                put(slot, rocrand_normal2(s));
                return true;
            }
            return false;
        case 10:
            if constexpr(has_normal4<S>::value)
            {
                put(slot, rocrand_normal4(s));
                return true;
            }
            return false;
        case 11: put(slot, rocrand_normal_double(s)); return true;
        case 12:
            if constexpr(has_normal_double2<S>::value)
            {
                put(slot, rocrand_normal_double2(s));
                return true;
            }
            return false;
        case 13:
            if constexpr(has_normal_double4<S>::value)
            {
                put(slot, rocrand_normal_double4(s));
                return true;
            }
            return false;
        case 14: put(slot, rocrand_log_normal(s, mf, sf)); return true;
        case 15:
            if constexpr(has_log_normal2<S>::value)
            {
                put(slot, rocrand_log_normal2(s, mf, sf));
                return true;
            }
            return false;
        case 16:
            if constexpr(has_log_normal4<S>::value)
            {
                put(slot, rocrand_log_normal4(s, mf, sf));
                return true;
            }
            return false;
        case 17: put(slot, rocrand_log_normal_double(s, md, sd)); return true;
        case 18:
            if constexpr(has_log_normal_double2<S>::value)
            {
                put(slot, rocrand_log_normal_double2(s, md, sd));
                return true;
            }
            return false;
        case 19:
            if constexpr(has_log_normal_double4<S>::value)
            {
                put(slot, rocrand_log_normal_double4(s, md, sd));
                return true;
            }
            return false;
        case 20: put(slot, rocrand_poisson(s, a.p0)); return true;
        case 21:
            if constexpr(has_poisson4<S>::value)
            {
                put(slot, rocrand_poisson4(s, a.p0));
                return true;
            }
            return false;
        case 22: put(slot, rocrand_discrete(s, dd)); return true;
        case 23:
            if constexpr(has_discrete4<S>::value)
            {
                put(slot, rocrand_discrete4(s, dd));
                return true;
            }
            return false;
        case 24: // skip ahead by p0 + c values, then one raw value
            if constexpr(has_skip<S>::value)
            {
                skipahead(static_cast<unsigned long long>(a.p0) + c, s);
                put(slot, rocrand(s));
                return true;
            }
            return false;
        case 25:
            if constexpr(has_skip_subsequence<S>::value)
            {
                skipahead_subsequence(static_cast<unsigned long long>(a.p0) + c, s);
                put(slot, rocrand(s));
                return true;
            }
            return false;
        case 26:
            if constexpr(has_skip_sequence<S>::value)
            {
                skipahead_sequence(static_cast<unsigned long long>(a.p0) + c, s);
                put(slot, rocrand(s));
                return true;
            }
            return false;
        case 27: // a mix that crosses the cached Box-Muller values
        {
            const int g = (c * 7 + 3) % 6;
            if(g == 0)
                put(slot, rocrand_normal(s));
            else if(g == 1)
                put(slot, rocrand_normal_double(s));
            else if(g == 2)
                put(slot, rocrand_log_normal(s, mf, sf));
            else if(g == 3)
                put(slot, rocrand_log_normal_double(s, md, sd));
            else if(g == 4)
                put(slot, rocrand_uniform(s));
            else
                put(slot, rocrand_poisson(s, 6000.0));
            return true;
        }
        default: return false;
    }
}

template<class S>
__device__ void init_pseudo(S* s, const Args& a, unsigned t)
{
    if constexpr(std::is_same_v<S, rocrand_state_lfsr113>)
    {
        const uint4 seed = make_uint4(static_cast<unsigned int>(a.seed), static_cast<unsigned int>(a.seed >> 32),
                                      static_cast<unsigned int>(a.seed) ^ 0x9e3779b9u,
                                      static_cast<unsigned int>(a.seed >> 32) ^ 0x7f4a7c15u);
        rocrand_init(seed, t, 7ull * t, s);
    }
    else
    {
        rocrand_init(a.seed, t, 7ull * t, s);
    }
}

template<class S>
__global__ void run_pseudo(Args a, int* unsupported)
{
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    S              s;
    init_pseudo(&s, a, t);
    for(int c = 0; c < a.calls; c++)
        if(!call(&s, a.func, c, a, a.out + (static_cast<size_t>(t) * a.calls + c) * 32))
            *unsupported = 1;
}

template<class S, class V>
__global__ void run_quasi(Args a, int* unsupported, bool scrambled)
{
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    S              s;
    if constexpr(std::is_same_v<S, rocrand_state_scrambled_sobol32>)
        rocrand_init(static_cast<const V*>(a.vec), static_cast<unsigned int>(a.scramble), 5u * t, &s);
    else if constexpr(std::is_same_v<S, rocrand_state_scrambled_sobol64>)
        rocrand_init(static_cast<const V*>(a.vec), static_cast<unsigned long long>(a.scramble), 5u * t, &s);
    else
        rocrand_init(static_cast<const V*>(a.vec), 5u * t, &s);
    for(int c = 0; c < a.calls; c++)
        if(!call(&s, a.func, c, a, a.out + (static_cast<size_t>(t) * a.calls + c) * 32))
            *unsupported = 1;
}

// MTGP32: one state per block copied into shared memory, every thread calling together;
// with func 28 the parameter set is taken again from a rocrand_make_constant table first
__global__ void run_mtgp32(Args a, int* unsupported, rocrand_state_mtgp32* states, mtgp32_params* consts)
{
    __shared__ rocrand_state_mtgp32 s;
    rocrand_mtgp32_block_copy(&states[blockIdx.x], &s);
    int func = a.func;
    if(func == 28)
    {
        if(threadIdx.x == 0)
            rocrand_mtgp32_set_params(&s, consts);
        __syncthreads();
        func = 0;
    }
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    for(int c = 0; c < a.calls; c++)
        if(!call(&s, func, c, a, a.out + (static_cast<size_t>(t) * a.calls + c) * 32))
            *unsupported = 1;
}

} // namespace

// devapi_run_mtgp32: `blocks` blocks of 256 threads, states made by rocrand_make_state_mtgp32
// from the published parameter sets and `seed`.
extern "C" int devapi_run_mtgp32(int func, unsigned long long seed, int blocks, int calls, double p0, double p1,
                                 const void* dist, void* out)
{
    Args a{func, calls, p0, p1, seed, nullptr, 0, static_cast<const rocrand_discrete_distribution_st*>(dist),
           static_cast<unsigned char*>(out)};
    int*                  flag   = nullptr;
    rocrand_state_mtgp32* states = nullptr;
    mtgp32_params*        consts = nullptr;
    int                   rc     = 2;
    if(cudaMalloc(&flag, sizeof(int)) == cudaSuccess
       && cudaMalloc(&states, sizeof(rocrand_state_mtgp32) * blocks) == cudaSuccess
       && cudaMalloc(&consts, sizeof(mtgp32_params)) == cudaSuccess
       && rocrand_make_state_mtgp32(states, mtgp32dc_params_fast_11213, blocks, seed) == ROCRAND_STATUS_SUCCESS
       && rocrand_make_constant(mtgp32dc_params_fast_11213, consts) == ROCRAND_STATUS_SUCCESS)
    {
        cudaMemset(flag, 0, sizeof(int));
        run_mtgp32<<<blocks, 256>>>(a, flag, states, consts);
        int unsupported = 0;
        if(cudaDeviceSynchronize() == cudaSuccess
           && cudaMemcpy(&unsupported, flag, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess)
            rc = unsupported ? 1 : 0;
    }
    cudaFree(flag);
    cudaFree(states);
    cudaFree(consts);
    return rc;
}

extern "C" int devapi_run(int engine, int func, unsigned long long seed, int threads, int calls, double p0,
                          double p1, const void* vec, unsigned long long scramble, const void* dist, void* out)
{
    Args a{func, calls, p0, p1, seed, vec, scramble, static_cast<const rocrand_discrete_distribution_st*>(dist),
           static_cast<unsigned char*>(out)};
    int* flag = nullptr;
    if(cudaMalloc(&flag, sizeof(int)) != cudaSuccess)
        return 2;
    cudaMemset(flag, 0, sizeof(int));
    const int block = 64, grid = (threads + block - 1) / block;
    switch(engine)
    {
        case 0: run_pseudo<rocrand_state_philox4x32_10><<<grid, block>>>(a, flag); break;
        case 1: run_pseudo<rocrand_state_mrg32k3a><<<grid, block>>>(a, flag); break;
        case 2: run_pseudo<rocrand_state_mrg31k3p><<<grid, block>>>(a, flag); break;
        case 3: run_pseudo<rocrand_state_threefry2x32_20><<<grid, block>>>(a, flag); break;
        case 4: run_pseudo<rocrand_state_threefry2x64_20><<<grid, block>>>(a, flag); break;
        case 5: run_pseudo<rocrand_state_threefry4x32_20><<<grid, block>>>(a, flag); break;
        case 6: run_pseudo<rocrand_state_threefry4x64_20><<<grid, block>>>(a, flag); break;
        case 7: run_quasi<rocrand_state_sobol32, unsigned int><<<grid, block>>>(a, flag, false); break;
        case 8: run_quasi<rocrand_state_scrambled_sobol32, unsigned int><<<grid, block>>>(a, flag, true); break;
        case 9: run_quasi<rocrand_state_sobol64, unsigned long long><<<grid, block>>>(a, flag, false); break;
        case 10:
            run_quasi<rocrand_state_scrambled_sobol64, unsigned long long><<<grid, block>>>(a, flag, true);
            break;
        case 11: run_pseudo<rocrand_state_xorwow><<<grid, block>>>(a, flag); break;
        case 12: run_pseudo<rocrand_state_lfsr113><<<grid, block>>>(a, flag); break;
        default: cudaFree(flag); return 2;
    }
    int unsupported = 0;
    if(cudaDeviceSynchronize() != cudaSuccess
       || cudaMemcpy(&unsupported, flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    {
        cudaFree(flag);
        return 2;
    }
    cudaFree(flag);
    return unsupported ? 1 : 0;
}
