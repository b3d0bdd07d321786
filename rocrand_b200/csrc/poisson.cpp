// poisson.cpp -- host-built Poisson tables (see poisson.hpp).
#include "poisson.hpp"

#include <cmath>
#include <cstring>
#include <memory>

namespace rb200
{

uint32_t poisson_capacity(double lambda)
{
    return static_cast<uint32_t>(2 * static_cast<size_t>(16.0 * (2.0 + std::sqrt(lambda))));
}

void poisson_probabilities_into(double lambda, double* p, uint32_t& size, uint32_t& offset)
{
    // Probabilities are evaluated outwards from floor(lambda) and stop where they drop
    // below 1e-12, then shifted to start at index 0 (poisson.hpp:110-161).
    const size_t capacity   = 2 * static_cast<size_t>(16.0 * (2.0 + std::sqrt(lambda)));
    const double p_epsilon  = 1e-12;
    const double log_lambda = std::log(lambda);
    const int    left       = static_cast<int>(std::floor(lambda)) - static_cast<int>(capacity / 2);
    for(size_t i = 0; i < capacity; i++)
        p[i] = 0.0;

    int lo = 0;
    for(int i = static_cast<int>(capacity / 2); i >= 0; i--)
    {
        const double x  = left + i;
        const double pp = std::exp(x * log_lambda - std::lgamma(x + 1.0) - lambda);
        if(pp < p_epsilon)
        {
            lo = i + 1;
            break;
        }
        p[i] = pp;
    }
    int hi = static_cast<int>(capacity) - 1;
    for(int i = static_cast<int>(capacity / 2) + 1; i < static_cast<int>(capacity); i++)
    {
        const double x  = left + i;
        const double pp = std::exp(x * log_lambda - std::lgamma(x + 1.0) - lambda);
        if(pp < p_epsilon)
        {
            hi = i - 1;
            break;
        }
        p[i] = pp;
    }
    for(int i = lo; i <= hi; i++)
        p[i - lo] = p[i];
    size   = static_cast<uint32_t>(hi - lo + 1);
    offset = static_cast<uint32_t>(left + lo);

    // normalize (discrete.hpp:189-205): sum in index order, then divide.
    double sum = 0.0;
    for(uint32_t i = 0; i < size; i++)
        sum += p[i];
    for(uint32_t i = 0; i < size; i++)
        p[i] /= sum;
}

void poisson_probabilities(double lambda, std::vector<double>& p, uint32_t& size, uint32_t& offset)
{
    p.assign(poisson_capacity(lambda), 0.0);
    poisson_probabilities_into(lambda, p.data(), size, offset);
}

void build_alias_into(double* p, uint32_t size, double* prob, uint32_t* alias, uint32_t* small,
                      uint32_t* large)
{
    // Vose's method with LIFO worklists; the pop order fixes which index becomes whose
    // alias, so it follows discrete.hpp:212-265 step for step.
    const double average = 1.0 / size;
    uint32_t     ns = 0, nl = 0;
    for(uint32_t i = 0; i < size; i++)
    {
        prob[i]  = 0.0;
        alias[i] = 0;
        if(p[i] >= average)
            large[nl++] = i;
        else
            small[ns++] = i;
    }
    while(ns > 0 && nl > 0)
    {
        const uint32_t less = small[--ns];
        const uint32_t more = large[--nl];
        prob[less]          = p[less] * size;
        alias[less]         = more;
        p[more]             = (p[more] + p[less]) - average;
        if(p[more] >= average)
            large[nl++] = more;
        else
            small[ns++] = more;
    }
    for(uint32_t i = 0; i < ns; i++)
        prob[small[i]] = 1.0;
    for(uint32_t i = 0; i < nl; i++)
        prob[large[i]] = 1.0;
}

void build_alias(const std::vector<double>& p_in, uint32_t size, std::vector<double>& prob,
                 std::vector<uint32_t>& alias)
{
    std::vector<double>   p(p_in.begin(), p_in.begin() + size);
    std::vector<uint32_t> small(size), large(size);
    prob.assign(size, 0.0);
    alias.assign(size, 0u);
    build_alias_into(p.data(), size, prob.data(), alias.data(), small.data(), large.data());
}

void build_cdf(const std::vector<double>& p, uint32_t size, std::vector<double>& cdf)
{
    cdf.assign(size, 0.0);
    double sum = 0.0;
    for(uint32_t i = 0; i < size; i++)
    {
        sum += p[i];
        cdf[i] = sum;
    }
}

void build_poisson_table(double lambda, HostPoissonTable& t)
{
    std::vector<double> p;
    poisson_probabilities(lambda, p, t.size, t.offset);
    build_alias(p, t.size, t.prob, t.alias);
    build_cdf(p, t.size, t.cdf);
}

namespace
{

// A table as kernel parameters (each struct stays under the 32 KB parameter limit).
struct PoissonEntriesUpload
{
    unsigned long long* thr;
    uint32_t*           alias;
    uint32_t            size;
    unsigned long long  thr_v[kPoissonTableCap];
    uint32_t            alias_v[kPoissonTableCap];
};

struct PoissonDoublesUpload
{
    double*  dst;
    uint32_t size;
    double   v[kPoissonTableCap];
};

__global__ void poisson_upload_entries(const __grid_constant__ PoissonEntriesUpload u)
{
    for(uint32_t i = threadIdx.x; i < u.size; i += blockDim.x)
    {
        u.thr[i]   = u.thr_v[i];
        u.alias[i] = u.alias_v[i];
    }
}

__global__ void poisson_upload_doubles(const __grid_constant__ PoissonDoublesUpload u)
{
    for(uint32_t i = threadIdx.x; i < u.size; i += blockDim.x)
        u.dst[i] = u.v[i];
}

// Host staging of the entries upload, one per calling thread (the kernel launch copies it).
thread_local PoissonEntriesUpload t_entries;

rocrand_status upload_doubles(double* dst, const std::vector<double>& v, uint32_t size, cudaStream_t stream)
{
    auto u  = std::make_unique<PoissonDoublesUpload>();
    u->dst  = dst;
    u->size = size;
    std::memcpy(u->v, v.data(), size * sizeof(double));
    poisson_upload_doubles<<<1, 256, 0, stream>>>(*u);
    return cudaGetLastError() == cudaSuccess ? ROCRAND_STATUS_SUCCESS : ROCRAND_STATUS_LAUNCH_FAILURE;
}

} // namespace

rocrand_status upload_alias_entries(unsigned long long* thr, uint32_t* alias_dst, const double* prob,
                                    const uint32_t* alias, uint32_t size, cudaStream_t stream)
{
    if(size > kPoissonTableCap)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    PoissonEntriesUpload& u = t_entries;
    u.thr                   = thr;
    u.alias                 = alias_dst;
    u.size                  = size;
    for(uint32_t i = 0; i < size; i++)
    {
        u.thr_v[i]   = alias_entry(prob[i], alias[i]);
        u.alias_v[i] = alias[i];
    }
    poisson_upload_entries<<<1, 256, 0, stream>>>(u);
    return cudaGetLastError() == cudaSuccess ? ROCRAND_STATUS_SUCCESS : ROCRAND_STATUS_LAUNCH_FAILURE;
}

PoissonCache::~PoissonCache()
{
    cudaFree(d_base);
}

rocrand_status PoissonCache::reserve()
{
    if(d_base != nullptr || m_host)
        return ROCRAND_STATUS_SUCCESS;
    static_assert(sizeof(PoissonEntriesUpload) < 32764 && sizeof(PoissonDoublesUpload) < 32764,
                  "kernel parameters are limited to 32764 bytes");
    const size_t cap = kPoissonTableCap;
    if(cudaMalloc(&d_base, cap * (3 * sizeof(double) + sizeof(uint32_t))) != cudaSuccess)
    {
        d_base = nullptr;
        return ROCRAND_STATUS_ALLOCATION_FAILED;
    }
    d_thr   = reinterpret_cast<unsigned long long*>(d_base);
    d_prob  = reinterpret_cast<double*>(d_base + cap * sizeof(double));
    d_cdf   = reinterpret_cast<double*>(d_base + 2 * cap * sizeof(double));
    d_alias = reinterpret_cast<uint32_t*>(d_base + 3 * cap * sizeof(double));
    return ROCRAND_STATUS_SUCCESS;
}

rocrand_status PoissonCache::get(double lambda, cudaStream_t stream, bool with_cdf, DistParams& p)
{
    if(lambda > kPoissonHugeLambda)
    {
        p.huge        = 1;
        p.lambda      = lambda;
        p.sqrt_lambda = std::sqrt(lambda);
        return ROCRAND_STATUS_SUCCESS;
    }
    if(m_host)
    {
        if(lambda != m_lambda || h_thr.empty())
        {
            build_poisson_table(lambda, h_table);
            h_thr.resize(h_table.size);
            for(uint32_t i = 0; i < h_table.size; i++)
                h_thr[i] = alias_entry(h_table.prob[i], h_table.alias[i]);
            m_lambda = lambda;
        }
        p.huge   = 0;
        p.prob   = h_table.prob.data();
        p.thr    = h_thr.data();
        p.alias  = h_table.alias.data();
        p.cdf    = h_table.cdf.data();
        p.size   = h_table.size;
        p.offset = h_table.offset;
        p.lambda = lambda;
        return ROCRAND_STATUS_SUCCESS;
    }
    rocrand_status st = reserve();
    if(st != ROCRAND_STATUS_SUCCESS)
        return st;
    if(lambda != m_lambda || (with_cdf && !m_has_cdf))
    {
        HostPoissonTable t;
        build_poisson_table(lambda, t);
        if(t.size > kPoissonTableCap)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        st = upload_alias_entries(d_thr, d_alias, t.prob.data(), t.alias.data(), t.size, stream);
        if(st == ROCRAND_STATUS_SUCCESS)
            st = upload_doubles(d_prob, t.prob, t.size, stream);
        if(st == ROCRAND_STATUS_SUCCESS && with_cdf)
            st = upload_doubles(d_cdf, t.cdf, t.size, stream);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        m_lambda  = lambda;
        m_has_cdf = with_cdf;
        m_size    = t.size;
        m_offset  = t.offset;
    }
    p.huge   = 0;
    p.prob   = d_prob;
    p.thr    = d_thr;
    p.alias  = d_alias;
    p.cdf    = d_cdf;
    p.size   = m_size;
    p.offset = m_offset;
    p.lambda = lambda;
    return ROCRAND_STATUS_SUCCESS;
}

} // namespace rb200
