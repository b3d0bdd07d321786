// Accuracy of rocrand_b200/csrc/precise_math.cuh (host build of the device header), measured
// against binary128 (libquadmath), with glibc's log/sin/cos measured the same way beside it.
// Prints one line per function: max error in ulp, results not correctly rounded, count.
#include "precise_math.cuh"

#include <quadmath.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <random>

static double ulp_err(double got, __float128 exact)
{
    const double e = static_cast<double>(exact);
    const double u = std::nextafter(std::fabs(e), INFINITY) - std::fabs(e);
    return static_cast<double>(((__float128)got - exact) / (__float128)u);
}

int main(int argc, char** argv)
{
    const long      n = argc > 1 ? std::atol(argv[1]) : 200000;
    std::mt19937_64 rng(42);
    double          max_log = 0, max_sin = 0, max_cos = 0, max_glog = 0, max_gsin = 0, max_gcos = 0;
    long            miss_log = 0, miss_sin = 0, miss_cos = 0, miss_logf = 0, miss_glog = 0, miss_gsin = 0;
    for(long t = 0; t < n; t++)
    {
        // log: the Box-Muller inputs (k + 1) 2^-53 and general normal numbers
        const uint64_t r = rng();
        const double   x = (t & 1) ? (static_cast<double>(r >> 11) + 1.0) * 0x1p-53
                                   : std::ldexp(1.0 + static_cast<double>(r >> 12) * 0x1p-52,
                                                static_cast<int>(r % 200) - 150);
        const __float128 lx = logq((__float128)x);
        const double     a = rb200::pm::log(x), g = std::log(x);
        max_log            = std::fmax(max_log, std::fabs(ulp_err(a, lx)));
        max_glog           = std::fmax(max_glog, std::fabs(ulp_err(g, lx)));
        miss_log += a != static_cast<double>(lx);
        miss_glog += g != static_cast<double>(lx);
        const float xf = static_cast<float>(x);
        if(xf > 0.0f)
            miss_logf += rb200::pm::logf(xf) != static_cast<float>(logq((__float128)xf));
        // sin/cos on (0, 2 pi]: the Box-Muller angles w * pi, w = k 2^-52
        const double ang = (static_cast<double>(rng() >> 11) + 1.0) * 0x1p-52 * 3.141592653589793;
        double       s, c;
        rb200::pm::sincos(ang, s, c);
        const __float128 es = sinq((__float128)ang), ec = cosq((__float128)ang);
        max_sin             = std::fmax(max_sin, std::fabs(ulp_err(s, es)));
        max_cos             = std::fmax(max_cos, std::fabs(ulp_err(c, ec)));
        max_gsin            = std::fmax(max_gsin, std::fabs(ulp_err(std::sin(ang), es)));
        max_gcos            = std::fmax(max_gcos, std::fabs(ulp_err(std::cos(ang), ec)));
        miss_sin += s != static_cast<double>(es);
        miss_cos += c != static_cast<double>(ec);
        miss_gsin += std::sin(ang) != static_cast<double>(es);
    }
    // log near 1 (where the result is small and the reduction must not cancel) and at both
    // sides of every table boundary, in three binades
    double max_near = 0;
    long   miss_near = 0, n_near = 0;
    auto   near = [&](double x) {
        const __float128 lx = logq((__float128)x);
        const double     a  = rb200::pm::log(x);
        max_near            = std::fmax(max_near, std::fabs(ulp_err(a, lx)));
        miss_near += a != static_cast<double>(lx);
        n_near++;
    };
    for(long k = 1; k <= 200000; k++)
    {
        near(1.0 + static_cast<double>(k) * 0x1p-52);
        near(1.0 - static_cast<double>(k) * 0x1p-53);
    }
    for(uint64_t i = 0; i < RB_LOG_ROWS; i++)
        for(int d = -3; d <= 3; d++)
        {
            double z;
            const uint64_t b = RB_LOG_OFF + (i << 44) + static_cast<uint64_t>(static_cast<int64_t>(d));
            std::memcpy(&z, &b, 8);
            near(z);
            near(z * 0.5);
            near(z * 1024.0);
        }
    std::printf("log %.6f %ld %ld\n", max_log, miss_log, n);
    std::printf("log_near %.6f %ld %ld\n", max_near, miss_near, n_near);
    std::printf("sin %.6f %ld %ld\n", max_sin, miss_sin, n);
    std::printf("cos %.6f %ld %ld\n", max_cos, miss_cos, n);
    std::printf("logf 0 %ld %ld\n", miss_logf, n);
    std::printf("glibc_log %.6f %ld %ld\n", max_glog, miss_glog, n);
    std::printf("glibc_sin %.6f %ld %ld\n", max_gsin, miss_gsin, n);
    // special values
    const double sp[] = {0.0, -0.0, -1.0, NAN, INFINITY, 4.9e-324, 1e-310, 1.0};
    for(double v : sp)
    {
        const double a = rb200::pm::log(v), g = std::log(v);
        const bool   same = (std::isnan(a) && std::isnan(g)) || a == g;
        std::printf("special %g %d\n", v, same ? 1 : 0);
    }
    return 0;
}
