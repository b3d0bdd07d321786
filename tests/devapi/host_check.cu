// host_check.cu -- the device API's functions run on the host (they are __host__ __device__):
// the inversion Poisson sampler over the lambdas whose segments rescale (300, 700, 999, 1200
// -- the last through the normal approximation), checked by the sample mean and variance.
// Prints "lambda mean var" per line.  TEST INFRASTRUCTURE ONLY.
#include <rocrand/rocrand_kernel.h>

#include <cstdio>

int main()
{
    const double lambdas[] = {3.5, 300.0, 700.0, 999.0, 1200.0};
    for(double lambda : lambdas)
    {
        rocrand_state_threefry4x32_20 s;
        rocrand_init(12345ull, 0, 0, &s);
        const int n   = 200000;
        double    sum = 0.0, sq = 0.0;
        for(int i = 0; i < n; i++)
        {
            const double k = rocrand_poisson(&s, lambda);
            sum += k;
            sq += k * k;
        }
        const double mean = sum / n;
        std::printf("%g %.6f %.6f\n", lambda, mean, sq / n - mean * mean);
    }
    return 0;
}
