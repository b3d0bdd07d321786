// poisson.hpp -- host-built Poisson tables, cached on the device per generator.
//
// The table (alias method) is built on the host with the same libm calls and the same
// operation order as the reference (library/src/rng/distribution/poisson.hpp:110-161 and
// discrete.hpp:189-265), because Poisson output must be bit-exact and depends on
// exp/lgamma of the host libm.  The device copy is refreshed in stream order when lambda
// changes, like poisson_distribution_manager::get_distribution (poisson.hpp:277-351): the
// new table travels as the parameters of a small upload kernel, so a call captured into a
// CUDA graph carries its own table, and the update needs no host memory that must outlive
// the call and no wait on earlier uploads.
#pragma once

#include "common.hpp"

#include <cmath>
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
// The same on caller storage: p must hold poisson_capacity(lambda) doubles.
void poisson_probabilities_into(double lambda, double* p, uint32_t& size, uint32_t& offset);

// Alias table (Vose, same stack order) and cumulative table of normalised p[0..size).
void build_alias(const std::vector<double>& p, uint32_t size, std::vector<double>& prob,
                 std::vector<uint32_t>& alias);
// The same on caller storage, allocating nothing: p[0..size) is consumed (overwritten),
// prob / alias receive the table, small / large are work lists of `size` entries each.
void build_alias_into(double* p, uint32_t size, double* prob, uint32_t* alias, uint32_t* small,
                      uint32_t* large);
void build_cdf(const std::vector<double>& p, uint32_t size, std::vector<double>& cdf);

// Builds the full table for lambda (prob, alias and cdf).
void build_poisson_table(double lambda, HostPoissonTable& t);

// The alias-table test of a 32-bit input r (discrete_alias, rocrand_discrete.h:38-63):
// x = r 2^-32, nx = size x, y = nx - floor(nx), pick i = floor(nx) when y < prob[i].  With
// r < 2^32 and size <= 4096 every step is exact, so i = (size r) >> 32 and y < prob[i] is
// ((size r) mod 2^32) < prob[i] 2^32, i.e. the low word below ceil(prob[i] 2^32): the kernels
// compare integers against these thresholds and pick the same entries.
inline unsigned long long alias_threshold(double prob)
{
    return prob >= 1.0 ? (1ull << 32) : static_cast<unsigned long long>(std::ceil(std::ldexp(prob, 32)));
}
// The kernels' table entry: threshold (33 bits) and alias (the rest) in one 64-bit word.
inline unsigned long long alias_entry(double prob, uint32_t alias)
{
    return alias_threshold(prob) | (static_cast<unsigned long long>(alias) << 33);
}

// Largest table: poisson_capacity(kPoissonHugeLambda) = 2 * floor(16 * (2 + sqrt(4000))).
constexpr uint32_t kPoissonTableCap = 2086;

// Writes packed entries (alias_entry of prob[i], alias[i]) to thr[0..size) and alias[i] to
// alias_dst[0..size) on `stream`.  The values travel as the parameters of one small kernel,
// so the update is stream-ordered, is recorded whole by a CUDA graph capture, and needs no
// host memory that outlives the call; the host staging is per calling thread.  size must
// not exceed kPoissonTableCap.
rocrand_status upload_alias_entries(unsigned long long* thr, uint32_t* alias_dst, const double* prob,
                                    const uint32_t* alias, uint32_t size, cudaStream_t stream);

// Per-generator device cache of the table for the most recent lambda.
class PoissonCache
{
public:
    PoissonCache() = default;
    ~PoissonCache();
    PoissonCache(const PoissonCache&)            = delete;
    PoissonCache& operator=(const PoissonCache&) = delete;

    // Allocates the device tables (once; generators call it from init(), as the reference's
    // generators initialise their Poisson manager, so that no allocation is left for a
    // generate call that a stream capture records).
    rocrand_status reserve();

    // Fills p with the distribution for lambda, uploading a new table on `stream` when
    // lambda changed.  with_cdf also uploads the cumulative table (used by Sobol).
    rocrand_status get(double lambda, cudaStream_t stream, bool with_cdf, DistParams& p);

    // Host execution: the tables stay in host memory (no device allocation or upload).
    void set_host() { m_host = true; }

private:
    bool                            m_host = false;
    std::vector<unsigned long long> h_thr;
    HostPoissonTable                h_table;
    double              m_lambda  = 0.0;
    bool                m_has_cdf = false;
    uint32_t            m_size = 0, m_offset = 0;
    unsigned char*      d_base  = nullptr; // one allocation for the four tables
    unsigned long long* d_thr   = nullptr; // packed alias entries (alias_entry)
    double*             d_prob  = nullptr;
    double*             d_cdf   = nullptr;
    uint32_t*           d_alias = nullptr;
};

} // namespace rb200
