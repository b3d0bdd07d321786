// poisson.cpp -- host-built Poisson tables (see poisson.hpp).
#include "poisson.hpp"

#include <cmath>
#include <cstring>

namespace rb200
{

uint32_t poisson_capacity(double lambda)
{
    return static_cast<uint32_t>(2 * static_cast<size_t>(16.0 * (2.0 + std::sqrt(lambda))));
}

void poisson_probabilities(double lambda, std::vector<double>& p, uint32_t& size, uint32_t& offset)
{
    // Probabilities are evaluated outwards from floor(lambda) and stop where they drop
    // below 1e-12, then shifted to start at index 0 (poisson.hpp:110-161).
    const size_t capacity   = 2 * static_cast<size_t>(16.0 * (2.0 + std::sqrt(lambda)));
    const double p_epsilon  = 1e-12;
    const double log_lambda = std::log(lambda);
    const int    left       = static_cast<int>(std::floor(lambda)) - static_cast<int>(capacity / 2);
    p.assign(capacity, 0.0);

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

void build_alias(const std::vector<double>& p_in, uint32_t size, std::vector<double>& prob,
                 std::vector<uint32_t>& alias)
{
    // Vose's method with LIFO worklists; the pop order fixes which index becomes whose
    // alias, so it follows discrete.hpp:212-265 step for step.
    std::vector<double> p(p_in.begin(), p_in.begin() + size);
    prob.assign(size, 0.0);
    alias.assign(size, 0u);
    const double          average = 1.0 / size;
    std::vector<uint32_t> small, large;
    small.reserve(size);
    large.reserve(size);
    for(uint32_t i = 0; i < size; i++)
        (p[i] >= average ? large : small).push_back(i);
    while(!small.empty() && !large.empty())
    {
        const uint32_t less = small.back();
        small.pop_back();
        const uint32_t more = large.back();
        large.pop_back();
        prob[less]  = p[less] * size;
        alias[less] = more;
        p[more]     = (p[more] + p[less]) - average;
        (p[more] >= average ? large : small).push_back(more);
    }
    for(uint32_t i : small)
        prob[i] = 1.0;
    for(uint32_t i : large)
        prob[i] = 1.0;
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

PoissonCache::~PoissonCache()
{
    if(m_upload)
    {
        cudaEventSynchronize(m_upload);
        cudaEventDestroy(m_upload);
    }
    cudaFree(d_prob);
    cudaFree(d_thr);
    cudaFree(d_alias);
    cudaFree(d_cdf);
    cudaFreeHost(h_prob);
    cudaFreeHost(h_thr);
    cudaFreeHost(h_alias);
    cudaFreeHost(h_cdf);
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
    if(m_cap == 0)
    {
        m_cap = poisson_capacity(kPoissonHugeLambda);
        if(cudaMalloc(&d_prob, m_cap * sizeof(double)) != cudaSuccess
           || cudaMalloc(&d_thr, m_cap * sizeof(unsigned long long)) != cudaSuccess
           || cudaMalloc(&d_alias, m_cap * sizeof(uint32_t)) != cudaSuccess
           || cudaMalloc(&d_cdf, m_cap * sizeof(double)) != cudaSuccess
           || cudaMallocHost(&h_prob, m_cap * sizeof(double)) != cudaSuccess
           || cudaMallocHost(&h_thr, m_cap * sizeof(unsigned long long)) != cudaSuccess
           || cudaMallocHost(&h_alias, m_cap * sizeof(uint32_t)) != cudaSuccess
           || cudaMallocHost(&h_cdf, m_cap * sizeof(double)) != cudaSuccess
           || cudaEventCreateWithFlags(&m_upload, cudaEventDisableTiming) != cudaSuccess)
        {
            m_cap = 0;
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        }
    }
    if(lambda != m_lambda || (with_cdf && !m_has_cdf))
    {
        HostPoissonTable t;
        build_poisson_table(lambda, t);
        // The staging buffers may still feed the previous upload.
        if(m_pending && cudaEventSynchronize(m_upload) != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        std::memcpy(h_prob, t.prob.data(), t.size * sizeof(double));
        for(uint32_t i = 0; i < t.size; i++)
            h_thr[i] = alias_entry(t.prob[i], t.alias[i]);
        std::memcpy(h_alias, t.alias.data(), t.size * sizeof(uint32_t));
        std::memcpy(h_cdf, t.cdf.data(), t.size * sizeof(double));
        if(cudaMemcpyAsync(d_prob, h_prob, t.size * sizeof(double), cudaMemcpyHostToDevice, stream)
               != cudaSuccess
           || cudaMemcpyAsync(d_thr, h_thr, t.size * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                              stream)
                  != cudaSuccess
           || cudaMemcpyAsync(d_alias, h_alias, t.size * sizeof(uint32_t), cudaMemcpyHostToDevice,
                              stream)
                  != cudaSuccess
           || cudaMemcpyAsync(d_cdf, h_cdf, t.size * sizeof(double), cudaMemcpyHostToDevice, stream)
                  != cudaSuccess
           || cudaEventRecord(m_upload, stream) != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        m_pending = true;
        m_lambda  = lambda;
        m_has_cdf = true;
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
