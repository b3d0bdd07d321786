/*
 * rocrand_discrete_types.h -- discrete distribution handle of the drop-in ABI.
 *
 * Same layout as the reference's library/include/rocrand/rocrand_discrete_types.h:30-50,
 * because callers (and device code built against the reference headers) read its fields
 * directly: size, offset, alias, probability, cdf in this order.
 */
#ifndef ROCRAND_DISCRETE_TYPES_H_
#define ROCRAND_DISCRETE_TYPES_H_

struct rocrand_discrete_distribution_st
{
    unsigned int  size;        /* number of entries in the tables */
    unsigned int  offset;      /* value of entry 0 */
    unsigned int* alias;       /* alias table (device memory) */
    double*       probability; /* alias-table probabilities (device memory) */
    double*       cdf;         /* cumulative distribution (device memory) */
};

typedef struct rocrand_discrete_distribution_st* rocrand_discrete_distribution;

#endif /* ROCRAND_DISCRETE_TYPES_H_ */
