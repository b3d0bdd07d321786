// Instantiates every engine and distribution of the reference's C++ wrapper
// (library/include/rocrand/rocrand.hpp) on this library's headers: rocrand.hpp includes
// rocrand/rocrand.h and rocrand/rocrand_kernel.h, which resolve to this library's copies, and
// every call it makes goes to librocrand.so.  Built and linked by tests/test_reference_wrapper.py;
// when run on a GPU it fills one small buffer through each engine x distribution and prints
// a checksum line per pair, or the error the wrapper raised (32-bit integers from a 64-bit
// quasi-random engine are a TYPE_ERROR in the reference too).
#include <rocrand/rocrand.hpp>

#include <cuda_runtime.h>

#include <cstdio>

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

static void* g_buf = nullptr;
static const size_t kN = 4096;

template<class T>
static unsigned long long sum_words(const T* dev, size_t n)
{
    static unsigned char host[kN * 8];
    cudaMemcpy(host, dev, n * sizeof(T), cudaMemcpyDeviceToHost);
    unsigned long long s = 0;
    for(size_t i = 0; i < n * sizeof(T); i++)
        s = s * 131 + host[i];
    return s;
}

template<class Engine>
static void fill_all(const char* name)
{
    try
    {
        Engine e;
        rc::uniform_int_distribution<unsigned int> ui;
        rc::uniform_real_distribution<float>       uf;
        rc::uniform_real_distribution<double>      ud;
        rc::normal_distribution<float>             nf(0.0f, 1.0f);
        rc::lognormal_distribution<double>         ld(0.0, 1.0);
        rc::poisson_distribution<unsigned int>     po(10.0);
        ui(e, static_cast<unsigned int*>(g_buf), kN);
        std::printf("%s uint %llu\n", name, sum_words(static_cast<unsigned int*>(g_buf), kN));
        uf(e, static_cast<float*>(g_buf), kN);
        std::printf("%s uniform_float %llu\n", name, sum_words(static_cast<float*>(g_buf), kN));
        ud(e, static_cast<double*>(g_buf), kN);
        std::printf("%s uniform_double %llu\n", name, sum_words(static_cast<double*>(g_buf), kN));
        nf(e, static_cast<float*>(g_buf), kN);
        std::printf("%s normal_float %llu\n", name, sum_words(static_cast<float*>(g_buf), kN));
        ld(e, static_cast<double*>(g_buf), kN);
        std::printf("%s log_normal_double %llu\n", name, sum_words(static_cast<double*>(g_buf), kN));
        po(e, static_cast<unsigned int*>(g_buf), kN);
        std::printf("%s poisson %llu\n", name, sum_words(static_cast<unsigned int*>(g_buf), kN));
    }
    catch(const rc::error& err)
    {
        std::printf("%s error %d %s\n", name, static_cast<int>(err.error_code()), err.what());
    }
}

int main()
{
    if(cudaMalloc(&g_buf, kN * 8) != cudaSuccess)
    {
        std::printf("no device\n");
        return 2;
    }
    fill_all<rc::philox4x32_10>("philox4x32_10");
    fill_all<rc::xorwow>("xorwow");
    fill_all<rc::mrg31k3p>("mrg31k3p");
    fill_all<rc::mrg32k3a>("mrg32k3a");
    fill_all<rc::mtgp32>("mtgp32");
    fill_all<rc::lfsr113>("lfsr113");
    fill_all<rc::mt19937>("mt19937");
    fill_all<rc::threefry2x32>("threefry2x32");
    fill_all<rc::threefry2x64>("threefry2x64");
    fill_all<rc::threefry4x32>("threefry4x32");
    fill_all<rc::threefry4x64>("threefry4x64");
    fill_all<rc::sobol32>("sobol32");
    fill_all<rc::scrambled_sobol32>("scrambled_sobol32");
    fill_all<rc::sobol64>("sobol64");
    fill_all<rc::scrambled_sobol64>("scrambled_sobol64");
    cudaFree(g_buf);
    return 0;
}
