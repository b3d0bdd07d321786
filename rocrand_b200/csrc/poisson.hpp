// poisson.hpp -- host-built Poisson tables, cached on the device per generator.
//
// The table (alias method) is built on the host with the same libm calls and the same
// operation order as the reference (library/src/rng/distribution/poisson.hpp:110-161 and
// discrete.hpp:189-265), because Poisson output must be bit-exact and depends on
// exp/lgamma of the host libm.  The device copy is refreshed in stream order when lambda
// changes, like poisson_distribution_manager::get_distribution (poisson.hpp:277-351).
#pragma once

#include "common.hpp"

#include <vector>

namespace rb200
{

// Lambda above which the normal approximation replaces the table (rocrand_poisson.h:53).
constexpr double kPoissonHugeLambda = 4000.0;

struct HostPoissonTable
{
    std::vector<double>   prob;
    std::vector<uint32_t> alias;
    std::vector<double>   cdf;
    uint32_t              size   = 0;
    uint32_t              offset = 0;
};

// Table capacity for lambda: 2 * floor(16 * (2 + sqrt(lambda))) (poisson.hpp:114).
uint32_t poisson_capacity(double lambda);

// Normalised probabilities, offset and size exactly as calculate_poisson_probabilities +
// normalize (poisson.hpp:110-161, discrete.hpp:189-205).
void poisson_probabilities(double lambda, std::vector<double>& p, uint32_t& size,
                           uint32_t& offset);

// Alias table (Vose, same stack order) and cumulative table of normalised p[0..size).
void build_alias(const std::vector<double>& p, uint32_t size, std::vector<double>& prob,
                 std::vector<uint32_t>& alias);
void build_cdf(const std::vector<double>& p, uint32_t size, std::vector<double>& cdf);

// Builds the full table for lambda (prob, alias and cdf).
void build_poisson_table(double lambda, HostPoissonTable& t);

// Per-generator device cache of the table for the most recent lambda.
class PoissonCache
{
public:
    PoissonCache() = default;
    ~PoissonCache();
    PoissonCache(const PoissonCache&)            = delete;
    PoissonCache& operator=(const PoissonCache&) = delete;

    // Fills p with the distribution for lambda, uploading a new table on `stream` when
    // lambda changed.  with_cdf also uploads the cumulative table (used by Sobol).
    rocrand_status get(double lambda, cudaStream_t stream, bool with_cdf, DistParams& p);

private:
    double       m_lambda  = 0.0;
    bool         m_has_cdf = false;
    uint32_t     m_cap     = 0;
    uint32_t     m_size = 0, m_offset = 0;
    double*      d_prob  = nullptr;
    uint32_t*    d_alias = nullptr;
    double*      d_cdf   = nullptr;
    double*      h_prob  = nullptr; // pinned staging
    uint32_t*    h_alias = nullptr;
    double*      h_cdf   = nullptr;
    cudaEvent_t  m_upload = nullptr;
    bool         m_pending = false;
};

} // namespace rb200
