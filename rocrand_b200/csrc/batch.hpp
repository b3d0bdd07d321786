// batch.hpp -- many generators in one launch: host side of the work-descriptor table.
//
// A batch is a list of requests; each request is what one rocrand_generate_* call writes
// (a fresh generator of that type, seed and offset, or a resident generator state).  The
// host turns each request into a descriptor (engine position, distribution parameters,
// output layout exactly as the plain call would lay it out) and cuts it into tiles; one
// persistent kernel then lets every block take the next tile from a global counter.
#pragma once

#include "common.hpp"
#include "counter_engines.cuh"
#include "generators.hpp"

#include <vector>

namespace rb200
{

enum BatchKind : uint32_t
{
    BK_PHILOX   = 0,
    BK_XORWOW   = 1,
    BK_MRG32K3A = 2,
    BK_SOBOL32  = 3,
    BK_COUNT    = 4
};

enum BatchDist : uint32_t
{
    BD_UINT     = 0,
    BD_FLOAT    = 1,
    BD_DOUBLE   = 2,
    BD_NORMAL_F = 3,
    BD_POISSON  = 4,
    BD_COUNT    = 5
};

// Position of the Philox output contract of one plain call (see philox.cu).
struct BatchPhilox
{
    PhiloxKeys keys;
    uint4      c0;
    uint32_t   s0, head, start0, tail;
    // aligned requests whose counters keep their upper words (vector j = block x0 + j):
    // rounds 1-2 of the words that do not vary precomputed, as in the plain fast kernel
    uint32_t   fast, x0;
    PhiloxLane lane;
};

// One request as the kernel sees it.
struct BatchReq
{
    uint32_t           kind, dist;
    unsigned char*     data;  // output base
    unsigned char*     vec;   // first aligned vector (Philox / stateful)
    unsigned long long n;     // elements
    unsigned long long vec_n; // Philox: 16-byte vectors; stateful: ow-vectors; Sobol: points
    unsigned long long tile0; // first global tile
    uint32_t           units; // vectors / slots / points per tile
    uint32_t           head, tail;
    // distribution
    float         mean, stddev;
    const double* prob;
    const unsigned long long* thr; // packed alias entries (poisson.hpp alias_entry)
    const uint32_t* alias;
    const double* cdf;
    uint32_t      tsize, toff, huge;
    double        lambda, sqrt_lambda;
    // engines
    BatchPhilox     philox;
    uint32_t        base[2][6]; // stateful: engines >= start / below start
    uint32_t        start;
    uint32_t*       arena;      // stateful resident state (nullptr: fresh, seeded from base)
    uint32_t        xseq;       // fresh XORWOW: index of its two base word sequences
    uint32_t        sobol_offset;
    const uint32_t* sobol_v;    // the 32 direction vectors of dimension 0
};

// Tile sizes and grid of one (kind, dist) pair, chosen by the autotuner.
struct BatchTuning
{
    uint32_t units[BK_COUNT][BD_COUNT];       // batches of fresh generators (autotuned)
    uint32_t serve_units[BK_COUNT][BD_COUNT]; // serving batches: resident states, mixed sizes
    uint32_t blocks_per_sm;
};

// Default tile sizes, replaced by rocrand_b200_autotune_batch on a device.
BatchTuning& batch_tuning();

// A request of the public ABI turned into descriptors; owns the device table.
class BatchPlan
{
public:
    ~BatchPlan();
    // Validates and lays out the requests (fresh generators); Poisson tables are made
    // resident on `stream`.
    rocrand_status build(const void* requests, size_t count, cudaStream_t stream);
    // Appends one already-built descriptor (resident generators, used by the server).
    void add(const BatchReq& r) { m_reqs.push_back(r); }
    // Drops the descriptors, keeping the device table for reuse.
    void clear() { m_reqs.clear(); }
    // Serving batches (resident states, latency-bound mixes) take the serving tile sizes.
    void set_serving(bool serving) { m_serving = serving; }
    // Allocates the device tables and the pinned staging buffer for batches of up to `reqs`
    // requests and `tiles` tiles now, and loads the kernel, so that the first batches neither
    // allocate nor wait for the module to load.
    rocrand_status reserve(size_t reqs, size_t tiles);
    // Assigns tiles and uploads the table on `stream`.
    rocrand_status upload(cudaStream_t stream);
    // Launches the persistent kernel (resets the tile counter first).
    rocrand_status launch(cudaStream_t stream);
    // Replays a captured graph of reset + launch (captured on first use).
    rocrand_status replay(cudaStream_t stream);
    size_t requests() const { return m_reqs.size(); }
    unsigned long long bytes() const { return m_bytes; }

private:
    std::vector<BatchReq> m_reqs;
    bool                  m_serving = false;
    std::vector<uint32_t> m_tile_req;         // request index of every tile
    uint32_t*             d_tile_req = nullptr;
    size_t                m_tile_cap = 0;
    std::vector<uint32_t> m_seq;              // word sequences of fresh XORWOW requests
    uint32_t*             d_seq     = nullptr;
    size_t                m_seq_cap = 0;      // words
    unsigned long long    m_tiles   = 0;
    unsigned long long    m_bytes   = 0;
    BatchReq*             d_reqs    = nullptr;
    unsigned long long*   d_next    = nullptr;
    size_t                m_cap     = 0;
    cudaGraphExec_t       m_exec    = nullptr;
    int                   m_device  = -1;
    // pinned copy of the three tables: from pageable memory cudaMemcpyAsync may hold the host
    // until the stream reaches the copy, i.e. until the work it is queued behind has run
    unsigned char*        h_stage     = nullptr;
    size_t                m_stage_cap = 0;
    cudaEvent_t           m_staged    = nullptr; // the last upload's copies have read h_stage
};

// Fills the distribution fields of a descriptor (Poisson tables are cached per lambda).
rocrand_status batch_set_dist(BatchReq& r, uint32_t dist, double p0, double p1, cudaStream_t stream);
// Output layout of one plain call (head, vectors, tail) for the request's kind and dist.
rocrand_status batch_layout(BatchReq& r, void* output, size_t n);
// Bytes per output element.
uint32_t batch_elem_size(uint32_t dist);
// Engine values consumed (iw) and outputs written (ow) per distribution call.
void batch_widths(uint32_t kind, uint32_t dist, unsigned& iw, unsigned& ow);

} // namespace rb200
