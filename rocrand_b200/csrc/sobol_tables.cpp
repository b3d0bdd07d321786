// sobol_tables.cpp -- Sobol direction vectors and scramble constants, and their C-ABI getters
// (library/src/rocrand.cpp:590-634).
//
// Every table is computed at first use from the embedded Joe-Kuo parameters
// (data/sobol_params.bin, see data/make_sobol_params.py) with the Joe-Kuo recurrence, in
// 32-bit (v_j = m_j << (31 - j)) and 64-bit (m_j << (63 - j)) form.  The reference's
// scrambled tables are the plain tables plus a constant on every word (640000 for 32-bit,
// 1280000 for 64-bit: tools/scrambled_sobol{32,64}_direction_vector_generator.cpp), and its
// scramble-constant tables are the first 20000 draws of std::uniform_int_distribution over
// a default-seeded std::mt19937 (tools/scrambled_sobol{32,64}_constants_generator.cpp).
#include "sobol_tables.hpp"

#include <cstring>
#include <mutex>
#include <random>

extern "C" const unsigned char rb200_sobol_params_begin[];
extern "C" const unsigned char rb200_sobol_params_end[];
extern "C" const unsigned char rb200_logf_replay_begin[];
extern "C" const unsigned char rb200_logf_replay_end[];

namespace rb200
{

namespace
{

struct BitReader
{
    const unsigned char* p;
    size_t               pos = 0;
    uint32_t             get(int n)
    {
        uint32_t v = 0;
        for(int i = 0; i < n; i++, pos++)
            v |= static_cast<uint32_t>((p[pos / 8] >> (pos % 8)) & 1u) << i;
        return v;
    }
};

template<class W>
void build(const std::vector<uint32_t>& s, const std::vector<uint32_t>& a,
           const std::vector<std::vector<uint32_t>>& m, std::vector<W>& out)
{
    constexpr int B = 8 * sizeof(W);
    out.assign(static_cast<size_t>(kSobolDims) * B, 0);
    for(int j = 0; j < B; j++)
        out[j] = W(1) << (B - 1 - j);
    for(unsigned d = 1; d < kSobolDims; d++)
    {
        W*             v  = &out[static_cast<size_t>(d) * B];
        const uint32_t sd = s[d];
        for(uint32_t j = 0; j < sd; j++)
            v[j] = static_cast<W>(m[d][j]) << (B - 1 - j);
        for(int j = static_cast<int>(sd); j < B; j++)
        {
            W x = v[j - sd] ^ (v[j - sd] >> sd);
            for(uint32_t k = 1; k < sd; k++)
                if((a[d] >> (sd - 1 - k)) & 1u)
                    x ^= v[j - k];
            v[j] = x;
        }
    }
}

} // namespace

const SobolTables& sobol_tables()
{
    static SobolTables    t;
    static std::once_flag once;
    std::call_once(once, [] {
        const unsigned char* blob = rb200_sobol_params_begin;
        if(std::memcmp(blob, "RBSOBOL1", 8) != 0)
            return;
        uint32_t dims = 0;
        std::memcpy(&dims, blob + 8, 4);
        if(dims != kSobolDims)
            return;
        std::vector<uint32_t>              s(kSobolDims, 0), a(kSobolDims, 0);
        std::vector<std::vector<uint32_t>> m(kSobolDims);
        BitReader                          br{blob + 12};
        for(unsigned d = 1; d < kSobolDims; d++)
        {
            s[d] = br.get(5);
            a[d] = br.get(static_cast<int>(s[d]) - 1);
            for(uint32_t j = 0; j < s[d]; j++)
                m[d].push_back(br.get(static_cast<int>(j) + 1));
        }
        build(s, a, m, t.v32);
        build(s, a, m, t.v64);
        t.sv32 = t.v32;
        for(auto& x : t.sv32)
            x += 640000u;
        t.sv64 = t.v64;
        for(auto& x : t.sv64)
            x += 1280000ull;
        std::mt19937                            g32;
        std::uniform_int_distribution<uint32_t> d32;
        for(unsigned k = 0; k < kSobolDims; k++)
            t.c32.push_back(d32(g32));
        std::mt19937                                      g64;
        std::uniform_int_distribution<unsigned long long> d64;
        for(unsigned k = 0; k < kSobolDims; k++)
            t.c64.push_back(d64(g64));
        t.ok = true;
    });
    return t;
}

const void* sobol_device_vectors(bool is64, bool scrambled)
{
    static std::mutex   mu;
    static const void*  cache[64][4] = {};
    const SobolTables&  t            = sobol_tables();
    if(!t.ok)
        return nullptr;
    const int                   dev = device_info().device;
    const int                   k   = (is64 ? 2 : 0) + (scrambled ? 1 : 0);
    std::lock_guard<std::mutex> lock(mu);
    if(cache[dev][k])
        return cache[dev][k];
    const void*  src   = is64 ? static_cast<const void*>(scrambled ? t.sv64.data() : t.v64.data())
                              : static_cast<const void*>(scrambled ? t.sv32.data() : t.v32.data());
    const size_t bytes = static_cast<size_t>(kSobolDims) * (is64 ? 64 * 8 : 32 * 4);
    void*        d     = nullptr;
    if(cudaMalloc(&d, bytes) != cudaSuccess)
        return nullptr;
    if(cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
    {
        cudaFree(d);
        return nullptr;
    }
    cache[dev][k] = d;
    return d;
}

bool logf_replay_device(lr::Table& out)
{
    static std::mutex mu;
    static lr::Table  cache[64];
    static bool       done[64] = {};
    const int         dev = device_info().device;
    std::lock_guard<std::mutex> lock(mu);
    if(!done[dev])
    {
        // header: magic, bucket shift, bucket count, log2 key buckets, members, reachable, 0
        const unsigned char* blob  = rb200_logf_replay_begin;
        const size_t         bytes = static_cast<size_t>(rb200_logf_replay_end - rb200_logf_replay_begin);
        uint32_t             h[6];
        if(bytes < 32 || std::memcmp(blob, "RBLOGF02", 8) != 0)
            return false;
        std::memcpy(h, blob + 8, sizeof(h));
        const size_t bound_bytes = static_cast<size_t>(h[1]) * 4;
        const size_t bound_pad   = (bound_bytes + 32 + 15) / 16 * 16 - 32;
        const size_t key_bytes   = (static_cast<size_t>(4) << h[2]) * 4;
        if(h[0] != static_cast<uint32_t>(lr::kBucketShift) || h[1] != lr::kBuckets || h[2] < 1 || h[2] > 28
           || bytes != 32 + bound_pad + key_bytes)
            return false;
        void* d = nullptr;
        if(cudaMalloc(&d, bound_pad + key_bytes) != cudaSuccess)
            return false;
        if(cudaMemcpy(d, blob + 32, bound_pad + key_bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        {
            cudaFree(d);
            return false;
        }
        cache[dev].bound        = static_cast<const uint32_t*>(d);
        cache[dev].keys         = reinterpret_cast<const uint4*>(static_cast<const unsigned char*>(d) + bound_pad);
        cache[dev].log2_buckets = h[2];
        done[dev]             = true;
    }
    out = cache[dev];
    return true;
}

} // namespace rb200

using namespace rb200;

extern "C" {

rocrand_status ROCRANDAPI rocrand_get_direction_vectors32(const unsigned int**         vectors,
                                                          rocrand_direction_vector_set set)
{
    const SobolTables& t = sobol_tables();
    if(!t.ok)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    switch(set)
    {
        case ROCRAND_DIRECTION_VECTORS_32_JOEKUO6: *vectors = t.v32.data(); return ROCRAND_STATUS_SUCCESS;
        case ROCRAND_SCRAMBLED_DIRECTION_VECTORS_32_JOEKUO6:
            *vectors = t.sv32.data();
            return ROCRAND_STATUS_SUCCESS;
        default: return ROCRAND_STATUS_OUT_OF_RANGE;
    }
}

rocrand_status ROCRANDAPI rocrand_get_direction_vectors64(const unsigned long long**   vectors,
                                                          rocrand_direction_vector_set set)
{
    const SobolTables& t = sobol_tables();
    if(!t.ok)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    switch(set)
    {
        case ROCRAND_DIRECTION_VECTORS_64_JOEKUO6: *vectors = t.v64.data(); return ROCRAND_STATUS_SUCCESS;
        case ROCRAND_SCRAMBLED_DIRECTION_VECTORS_64_JOEKUO6:
            *vectors = t.sv64.data();
            return ROCRAND_STATUS_SUCCESS;
        default: return ROCRAND_STATUS_OUT_OF_RANGE;
    }
}

rocrand_status ROCRANDAPI rocrand_get_scramble_constants32(const unsigned int** constants)
{
    const SobolTables& t = sobol_tables();
    if(!t.ok)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    *constants = t.c32.data();
    return ROCRAND_STATUS_SUCCESS;
}

rocrand_status ROCRANDAPI rocrand_get_scramble_constants64(const unsigned long long** constants)
{
    const SobolTables& t = sobol_tables();
    if(!t.ok)
        return ROCRAND_STATUS_INTERNAL_ERROR;
    *constants = t.c64.data();
    return ROCRAND_STATUS_SUCCESS;
}

} // extern "C"
