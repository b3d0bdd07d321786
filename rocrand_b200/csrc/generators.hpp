// generators.hpp -- generator objects behind the C ABI, one class per engine family.
#pragma once

#include "common.hpp"
#include "counter_engines.cuh"
#include "poisson.hpp"

namespace rb200
{

// Common state of pseudo-random generators: seed, offset and ordering, with the
// reference's lazy re-initialisation on any change (generator_type.hpp:235-291).
class PseudoGeneratorBase : public rocrand_generator_base_type
{
public:
    rocrand_status set_seed(unsigned long long seed) override
    {
        m_seed        = seed;
        m_initialized = false;
        return ROCRAND_STATUS_SUCCESS;
    }
    rocrand_status set_offset(unsigned long long offset) override
    {
        m_offset      = offset;
        m_initialized = false;
        return ROCRAND_STATUS_SUCCESS;
    }

protected:
    // Host execution for a family that has a CPU form: tables stay on the host.
    bool enable_host()
    {
        m_host_exec = true;
        m_poisson.set_host();
        return true;
    }

    unsigned long long m_seed        = 0;
    unsigned long long m_offset      = 0;
    rocrand_ordering   m_order       = ROCRAND_ORDERING_PSEUDO_DEFAULT;
    bool               m_initialized = false;
    PoissonCache       m_poisson;
};

class PhiloxGenerator final : public PseudoGeneratorBase
{
public:
    PhiloxGenerator();
    ~PhiloxGenerator() override;
    rocrand_rng_type type() const override { return ROCRAND_RNG_PSEUDO_PHILOX4_32_10; }
    rocrand_status   init() override;
    rocrand_status   set_output_position(rb200::Dist d, unsigned long long index) override;
    rocrand_status   set_order(rocrand_ordering order) override;
    rocrand_status   generate(void* data, size_t n, Dist d, const DistParams& p) override;
    rocrand_status   generate_poisson(unsigned int* data, size_t n, double lambda) override;
    rocrand_status   batch_descriptor(uint32_t dist, double p0, double p1, void* data, size_t n,
                                      BatchReq& r, cudaStream_t stream) override;
    bool             set_host_execution() override { return enable_host(); }

private:
    CounterPos m_pos;
};

// Poisson values of a fresh Philox4x32-10 stream with a caller-supplied table (philox.cu).
rocrand_status philox_poisson_with_table(unsigned long long seed, unsigned long long offset,
                                         unsigned int* data, size_t n, const DistParams& p,
                                         cudaStream_t stream);

// Stateful engine families (stateful.cu, batch.cu).
enum class StatefulFamily
{
    XORWOW,
    MRG32K3A,
    MRG31K3P,
    LFSR113
};

// Engine states a fresh stateful generator (seed, offset) starts from: engines
// e >= start begin at base[0], engines below it at base[1]; engine e then jumps e
// subsequences with the per-digit tables.  LFSR113 takes its default uint4 seed here.
struct StatefulBases
{
    uint32_t base[2][6];
    uint32_t start;
};
StatefulBases stateful_bases(StatefulFamily fam, unsigned long long seed, unsigned long long offset);
// Per-digit subsequence jump tables of a family on the current device (uploaded once).
const void* stateful_digit_tables(StatefulFamily fam);
// XORWOW jump polynomials of the E engines (word-major, uploaded once per device).
const uint32_t* stateful_xorwow_jump_polys();
// The 164-word sequence s_0..s_163 continued from a base state's words 0..4.
void xorwow_word_sequence(const uint32_t* base, uint32_t* seq);

// Generator of any type (api.cpp); nullptr for an unknown type.
rocrand_generator_base_type* make_generator(rocrand_rng_type t);
// A host generator: the device generator of type t writing through to host memory.
rocrand_generator_base_type* make_host_generator(rocrand_rng_type t);

// Factories of the other generator families (one translation unit each).
rocrand_generator_base_type* make_threefry(rocrand_rng_type t);
rocrand_generator_base_type* make_stateful(rocrand_rng_type t);
rocrand_generator_base_type* make_mt19937();
rocrand_generator_base_type* make_mtgp32();
rocrand_generator_base_type* make_sobol(rocrand_rng_type t);

} // namespace rb200
