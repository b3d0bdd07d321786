// sobol_tables.hpp -- Sobol direction vectors (computed from the Joe-Kuo parameters).
#pragma once

#include "common.hpp"
#include "logf_replay.cuh"

#include <vector>

namespace rb200
{

constexpr unsigned kSobolDims = 20000;

struct SobolTables
{
    bool                            ok = false;
    std::vector<uint32_t>           v32, sv32; // kSobolDims x 32, plain / scrambled
    std::vector<unsigned long long> v64, sv64; // kSobolDims x 64
    std::vector<uint32_t>           c32;       // scramble constants (getter only)
    std::vector<unsigned long long> c64;
};

// Host tables, built once per process.
const SobolTables& sobol_tables();

// Device copy of one table on the current device (uploaded once per device).
const void* sobol_device_vectors(bool is64, bool scrambled);

// The host-logf replay table of the inverse-erf normal (logf_replay.cuh) on the current
// device, uploaded once per device; false if it is missing or could not be uploaded.
bool logf_replay_device(lr::Table& out);

} // namespace rb200
