// Instantiates every engine and distribution of the reference's C++ wrapper
// (library/include/rocrand/rocrand.hpp) on this library's headers: rocrand.hpp includes
// rocrand/rocrand.h and rocrand/rocrand_kernel.h, which resolve to this library's copies, and
// every call it makes goes to librocrand.so.  Built and linked by tests/test_reference_wrapper.py
// (and by __graft_entry__.build() into oracle/_ref/wrapper/, test infrastructure); run on a
// GPU by tests/test_reference_wrapper_gpu.py, it checks every engine x distribution of the
// wrapper against the same calls made through the C ABI.
#include <rocrand/rocrand.hpp>

#include <cuda_runtime.h>

#include <cstdio>
#include <type_traits>

namespace rc = rocrand_cpp;

template class rc::philox4x32_10_engine<>;
template class rc::xorwow_engine<>;
template class rc::mrg31k3p_engine<>;
template class rc::mrg32k3a_engine<>;
template class rc::mtgp32_engine<>;
template class rc::lfsr113_engine<>;
template class rc::mt19937_engine<>;
template class rc::threefry2x32_20_engine<>;
template class rc::threefry2x64_20_engine<>;
template class rc::threefry4x32_20_engine<>;
template class rc::threefry4x64_20_engine<>;
template class rc::sobol32_engine<>;
template class rc::scrambled_sobol32_engine<>;
template class rc::sobol64_engine<>;
template class rc::scrambled_sobol64_engine<>;
template class rc::uniform_int_distribution<unsigned char>;
template class rc::uniform_int_distribution<unsigned short>;
template class rc::uniform_int_distribution<unsigned int>;
template class rc::uniform_int_distribution<unsigned long long>;
template class rc::uniform_real_distribution<float>;
template class rc::uniform_real_distribution<double>;
template class rc::uniform_real_distribution<half>;
template class rc::normal_distribution<float>;
template class rc::normal_distribution<double>;
template class rc::normal_distribution<half>;
template class rc::lognormal_distribution<float>;
template class rc::lognormal_distribution<double>;
template class rc::lognormal_distribution<half>;
template class rc::poisson_distribution<unsigned int>;

static void*        g_buf = nullptr; // the wrapper's output
static void*        g_ref = nullptr; // the same call through the C ABI
static const size_t kN    = 4099;    // odd: head and tail paths of the kernels

static bool same(size_t bytes)
{
    static unsigned char a[kN * 8], b[kN * 8];
    cudaMemcpy(a, g_buf, bytes, cudaMemcpyDeviceToHost);
    cudaMemcpy(b, g_ref, bytes, cudaMemcpyDeviceToHost);
    for(size_t i = 0; i < bytes; i++)
        if(a[i] != b[i])
            return false;
    return true;
}

template<class E, class = void>
struct has_seed : std::false_type
{};
template<class E>
struct has_seed<E, std::void_t<typename E::seed_type>> : std::true_type
{};

// The plain generator seeded as the wrapper's default-constructed engine is (quasi-random
// engines have no seed: one dimension, offset 0, as a fresh generator).
template<class Engine>
static void seed_plain(rocrand_generator g)
{
    if constexpr(has_seed<Engine>::value)
    {
        if constexpr(std::is_same<typename Engine::seed_type, uint4>::value)
            rocrand_set_seed_uint4(g, Engine::default_seed);
        else
            rocrand_set_seed(g, Engine::default_seed);
    }
}

// Each distribution object of the wrapper fills g_buf through engine e; the same call on a
// plain generator of the same type, seeded as the wrapper seeds it, fills g_ref; the two
// must be byte-identical.  Prints "<engine> <distribution> OK|MISMATCH" or the wrapper's
// error (32-bit outputs from a 64-bit quasi-random engine are a TYPE_ERROR in the
// reference too).
template<class Engine>
static void fill_all(const char* name, rocrand_rng_type type)
{
    try
    {
        Engine            e;
        rocrand_generator g = nullptr;
        if(rocrand_create_generator(&g, type) != ROCRAND_STATUS_SUCCESS)
        {
            std::printf("%s create failed\n", name);
            return;
        }
        seed_plain<Engine>(g);
        rc::uniform_int_distribution<unsigned int> ui;
        rc::uniform_real_distribution<float>       uf;
        rc::uniform_real_distribution<double>      ud;
        rc::normal_distribution<float>             nf(0.0f, 1.0f);
        rc::lognormal_distribution<double>         ld(0.0, 1.0);
        rc::poisson_distribution<unsigned int>     po(10.0);
        auto report = [&](const char* dist, rocrand_status st, size_t bytes) {
            cudaDeviceSynchronize();
            std::printf("%s %s %s\n", name, dist,
                        st != ROCRAND_STATUS_SUCCESS ? "C-ABI-ERROR" : (same(bytes) ? "OK" : "MISMATCH"));
        };
        ui(e, static_cast<unsigned int*>(g_buf), kN);
        report("uint", rocrand_generate(g, static_cast<unsigned int*>(g_ref), kN), kN * 4);
        uf(e, static_cast<float*>(g_buf), kN);
        report("uniform_float", rocrand_generate_uniform(g, static_cast<float*>(g_ref), kN), kN * 4);
        ud(e, static_cast<double*>(g_buf), kN);
        report("uniform_double", rocrand_generate_uniform_double(g, static_cast<double*>(g_ref), kN), kN * 8);
        nf(e, static_cast<float*>(g_buf), kN - 1);
        report("normal_float", rocrand_generate_normal(g, static_cast<float*>(g_ref), kN - 1, 0.0f, 1.0f),
               (kN - 1) * 4);
        ld(e, static_cast<double*>(g_buf), kN - 1);
        report("log_normal_double",
               rocrand_generate_log_normal_double(g, static_cast<double*>(g_ref), kN - 1, 0.0, 1.0),
               (kN - 1) * 8);
        po(e, static_cast<unsigned int*>(g_buf), kN);
        report("poisson", rocrand_generate_poisson(g, static_cast<unsigned int*>(g_ref), kN, 10.0), kN * 4);
        rocrand_destroy_generator(g);
    }
    catch(const rc::error& err)
    {
        std::printf("%s error %d %s\n", name, static_cast<int>(err.error_code()), err.what());
    }
}

int main()
{
    if(cudaMalloc(&g_buf, kN * 8) != cudaSuccess || cudaMalloc(&g_ref, kN * 8) != cudaSuccess)
    {
        std::printf("no device\n");
        return 2;
    }
    fill_all<rc::philox4x32_10>("philox4x32_10", ROCRAND_RNG_PSEUDO_PHILOX4_32_10);
    fill_all<rc::xorwow>("xorwow", ROCRAND_RNG_PSEUDO_XORWOW);
    fill_all<rc::mrg31k3p>("mrg31k3p", ROCRAND_RNG_PSEUDO_MRG31K3P);
    fill_all<rc::mrg32k3a>("mrg32k3a", ROCRAND_RNG_PSEUDO_MRG32K3A);
    fill_all<rc::mtgp32>("mtgp32", ROCRAND_RNG_PSEUDO_MTGP32);
    fill_all<rc::lfsr113>("lfsr113", ROCRAND_RNG_PSEUDO_LFSR113);
    fill_all<rc::mt19937>("mt19937", ROCRAND_RNG_PSEUDO_MT19937);
    fill_all<rc::threefry2x32>("threefry2x32", ROCRAND_RNG_PSEUDO_THREEFRY2_32_20);
    fill_all<rc::threefry2x64>("threefry2x64", ROCRAND_RNG_PSEUDO_THREEFRY2_64_20);
    fill_all<rc::threefry4x32>("threefry4x32", ROCRAND_RNG_PSEUDO_THREEFRY4_32_20);
    fill_all<rc::threefry4x64>("threefry4x64", ROCRAND_RNG_PSEUDO_THREEFRY4_64_20);
    fill_all<rc::sobol32>("sobol32", ROCRAND_RNG_QUASI_SOBOL32);
    fill_all<rc::scrambled_sobol32>("scrambled_sobol32", ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL32);
    fill_all<rc::sobol64>("sobol64", ROCRAND_RNG_QUASI_SOBOL64);
    fill_all<rc::scrambled_sobol64>("scrambled_sobol64", ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL64);
    cudaFree(g_buf);
    cudaFree(g_ref);
    return 0;
}
