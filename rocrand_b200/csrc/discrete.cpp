// discrete.cpp -- discrete-distribution objects of the C ABI.
//
// rocrand_create_poisson_distribution / rocrand_create_discrete_distribution /
// rocrand_destroy_discrete_distribution (library/src/rocrand.cpp:451-588).  As in the
// reference, the returned handle is DEVICE memory holding a
// rocrand_discrete_distribution_st whose table pointers are device memory too, so device
// code can read it directly; tables hold both the alias and the CDF form
// (DISCRETE_METHOD_UNIVERSAL, discrete.hpp:79-117).
#include "common.hpp"
#include "poisson.hpp"

#include <vector>

namespace
{

rocrand_status upload_distribution(const std::vector<double>& p, uint32_t size, uint32_t offset,
                                   rocrand_discrete_distribution* out)
{
    using namespace rb200;
    std::vector<double>   prob;
    std::vector<uint32_t> alias;
    std::vector<double>   cdf;
    build_alias(p, size, prob, alias);
    build_cdf(p, size, cdf);

    rocrand_discrete_distribution_st h{};
    h.size   = size;
    h.offset = offset;
    if(cudaMalloc(&h.probability, sizeof(double) * size) != cudaSuccess
       || cudaMalloc(&h.alias, sizeof(uint32_t) * size) != cudaSuccess
       || cudaMalloc(&h.cdf, sizeof(double) * size) != cudaSuccess)
    {
        cudaFree(h.probability);
        cudaFree(h.alias);
        cudaFree(h.cdf);
        return ROCRAND_STATUS_ALLOCATION_FAILED;
    }
    if(cudaMemcpy(h.probability, prob.data(), sizeof(double) * size, cudaMemcpyHostToDevice)
           != cudaSuccess
       || cudaMemcpy(h.alias, alias.data(), sizeof(uint32_t) * size, cudaMemcpyHostToDevice)
              != cudaSuccess
       || cudaMemcpy(h.cdf, cdf.data(), sizeof(double) * size, cudaMemcpyHostToDevice)
              != cudaSuccess)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    if(cudaMalloc(out, sizeof(rocrand_discrete_distribution_st)) != cudaSuccess)
        return ROCRAND_STATUS_ALLOCATION_FAILED;
    if(cudaMemcpy(*out, &h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    return ROCRAND_STATUS_SUCCESS;
}

} // namespace

extern "C" {

rocrand_status ROCRANDAPI rocrand_create_poisson_distribution(
    double lambda, rocrand_discrete_distribution* discrete_distribution)
{
    if(discrete_distribution == nullptr || !(lambda > 0.0)) // lambda <= 0 (and NaN)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        std::vector<double> p;
        uint32_t            size = 0, offset = 0;
        rb200::poisson_probabilities(lambda, p, size, offset);
        return upload_distribution(p, size, offset, discrete_distribution);
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

rocrand_status ROCRANDAPI
    rocrand_create_discrete_distribution(const double*                  probabilities,
                                         unsigned int                   size,
                                         unsigned int                   offset,
                                         rocrand_discrete_distribution* discrete_distribution)
{
    if(discrete_distribution == nullptr || size == 0)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        // normalize (discrete.hpp:189-205), then the same table builders.
        std::vector<double> p(probabilities, probabilities + size);
        double              sum = 0.0;
        for(unsigned i = 0; i < size; i++)
            sum += p[i];
        for(unsigned i = 0; i < size; i++)
            p[i] /= sum;
        return upload_distribution(p, size, offset, discrete_distribution);
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

rocrand_status ROCRANDAPI
    rocrand_destroy_discrete_distribution(rocrand_discrete_distribution discrete_distribution)
{
    if(discrete_distribution == nullptr)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    rocrand_discrete_distribution_st h{};
    if(cudaMemcpy(&h, discrete_distribution, sizeof(h), cudaMemcpyDefault) != cudaSuccess)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    if(cudaFree(h.probability) != cudaSuccess || cudaFree(h.alias) != cudaSuccess
       || cudaFree(h.cdf) != cudaSuccess || cudaFree(discrete_distribution) != cudaSuccess)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    return ROCRAND_STATUS_SUCCESS;
}

} // extern "C"
