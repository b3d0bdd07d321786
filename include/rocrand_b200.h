/*
 * rocrand_b200.h -- entry points of librocrand that extend the rocRAND C ABI.
 *
 * Everything in include/rocrand/rocrand.h keeps the reference's meaning; the functions
 * below are additions of this library.
 */
#ifndef ROCRAND_B200_H_
#define ROCRAND_B200_H_

#include "rocrand/rocrand.h"

#if defined(__cplusplus)
extern "C" {
#endif

/*
 * Poisson values that need no device allocation.  No counterpart in the reference.
 *
 * Writes the n values that a fresh ROCRAND_RNG_PSEUDO_PHILOX4_32_10 generator with this
 * seed and offset would write with rocrand_generate_poisson(output_data, n, lambda) on
 * `stream`, without allocating anything: for callers that cannot call cudaMalloc (inside a
 * CUDA graph capture or a driver callback, or with device memory fully pre-partitioned).
 * Its scratch (the alias table of lambda, up to 4096 entries) is a fixed 48 KiB array that
 * every GPU loading the library holds until the process exits; lambda <= 0, NaN and tables
 * beyond 4096 entries give ROCRAND_STATUS_OUT_OF_RANGE.  The first call on a device, whatever
 * its lambda, looks up the array's address and should come before any stream capture.  Each
 * call writes its table into the array in stream order through a kernel's parameters, so a
 * call recorded by a graph capture carries its own table.  All calls share the array: calls
 * that overlap on the GPU race.  "Nothing" means device memory: no cudaMalloc or cudaFree is
 * made; the host staging of the table is a per-thread block of the library.
 */
rocrand_status ROCRANDAPI rocrand_b200_generate_poisson_noalloc(unsigned long long seed,
                                                                unsigned long long offset,
                                                                unsigned int*      output_data,
                                                                size_t             n,
                                                                double             lambda,
                                                                hipStream_t        stream);

/*
 * Output position, for sharding one stream over several GPUs or processes.  No counterpart
 * in the reference.
 *
 * The outputs of one rocrand_generate_* call of kind `output` are positioned at `index` of
 * the stream that a fresh generator of the same type and seed writes with that kind in one
 * call from offset 0: after this call, the next call of that kind writes exactly outputs
 * [index, index + n) of that single stream (into an output aligned like the single call's).
 * Rank r of N, each calling it with index = r * n before generating n outputs, therefore
 * writes slice r of one stream, with no communication.
 *  - XORWOW, MRG32k3a, MRG31k3p, LFSR113: output vector V = index / w (w outputs of iw
 *    engine values each, per the distribution) was served by engine V mod 131072, so every
 *    engine e is placed after iw * (V / 131072 + (e < V mod 131072)) values and the engine
 *    rotation starts at V mod 131072 -- a placement rocrand_set_offset cannot express when
 *    iw > 1 or w > 1 (uniform double, normal and log-normal outputs);
 *  - Philox4x32-10 and ThreeFry: the offset index / w * iw (rocrand_set_offset);
 *  - MT19937, MTGP32 and the quasi-random generators: ROCRAND_STATUS_TYPE_ERROR (they have
 *    no offset);
 * index not a multiple of w gives ROCRAND_STATUS_LENGTH_NOT_MULTIPLE.  The position replaces
 * any offset; a later rocrand_set_offset replaces the position.
 */
typedef enum rocrand_b200_output
{
    ROCRAND_B200_OUTPUT_UINT              = 0,  /* rocrand_generate */
    ROCRAND_B200_OUTPUT_UCHAR             = 1,  /* rocrand_generate_char */
    ROCRAND_B200_OUTPUT_USHORT            = 2,  /* rocrand_generate_short */
    ROCRAND_B200_OUTPUT_ULONGLONG         = 3,  /* rocrand_generate_long_long */
    ROCRAND_B200_OUTPUT_UNIFORM_FLOAT     = 4,  /* rocrand_generate_uniform */
    ROCRAND_B200_OUTPUT_UNIFORM_DOUBLE    = 5,  /* rocrand_generate_uniform_double */
    ROCRAND_B200_OUTPUT_UNIFORM_HALF      = 6,  /* rocrand_generate_uniform_half */
    ROCRAND_B200_OUTPUT_NORMAL_FLOAT      = 7,  /* rocrand_generate_normal */
    ROCRAND_B200_OUTPUT_NORMAL_DOUBLE     = 8,  /* rocrand_generate_normal_double */
    ROCRAND_B200_OUTPUT_NORMAL_HALF       = 9,  /* rocrand_generate_normal_half */
    ROCRAND_B200_OUTPUT_LOG_NORMAL_FLOAT  = 10, /* rocrand_generate_log_normal */
    ROCRAND_B200_OUTPUT_LOG_NORMAL_DOUBLE = 11, /* rocrand_generate_log_normal_double */
    ROCRAND_B200_OUTPUT_LOG_NORMAL_HALF   = 12, /* rocrand_generate_log_normal_half */
    ROCRAND_B200_OUTPUT_POISSON           = 13  /* rocrand_generate_poisson */
} rocrand_b200_output;

rocrand_status ROCRANDAPI rocrand_b200_set_output_position(rocrand_generator   generator,
                                                           rocrand_b200_output output,
                                                           unsigned long long  index);

/*
 * Batched fill.  No counterpart in the reference.
 *
 * A request is exactly one plain generate call on a fresh generator: rng_type created,
 * seeded with `seed` (ignored by QUASI_SOBOL32, which has one dimension here), set to
 * `offset`, then rocrand_generate (UINT), rocrand_generate_uniform (UNIFORM_FLOAT),
 * rocrand_generate_uniform_double (UNIFORM_DOUBLE), rocrand_generate_normal (NORMAL_FLOAT,
 * mean = param0, stddev = param1) or rocrand_generate_poisson (POISSON, lambda = param0)
 * into `output` (device memory, n elements).  The values written are those of that plain
 * call, bit for bit for UINT/UNIFORM/POISSON and identically computed for NORMAL.
 * rng_type is ROCRAND_RNG_PSEUDO_PHILOX4_32_10, ROCRAND_RNG_PSEUDO_XORWOW (or DEFAULT),
 * ROCRAND_RNG_PSEUDO_MRG32K3A or ROCRAND_RNG_QUASI_SOBOL32 (or QUASI_DEFAULT); anything else
 * gives ROCRAND_STATUS_TYPE_ERROR.  All requests of a batch run in one persistent kernel.
 */
typedef enum rocrand_b200_distribution
{
    ROCRAND_B200_DIST_UINT           = 0,
    ROCRAND_B200_DIST_UNIFORM_FLOAT  = 1,
    ROCRAND_B200_DIST_UNIFORM_DOUBLE = 2,
    ROCRAND_B200_DIST_NORMAL_FLOAT   = 3,
    ROCRAND_B200_DIST_POISSON        = 4
} rocrand_b200_distribution;

typedef struct rocrand_b200_request
{
    rocrand_rng_type          rng_type;
    rocrand_b200_distribution distribution;
    unsigned long long        seed;
    unsigned long long        offset;
    double                    param0;
    double                    param1;
    void*                     output;
    size_t                    n;
} rocrand_b200_request;

/* Runs `count` requests in one launch on `stream` and waits for it. */
rocrand_status ROCRANDAPI rocrand_b200_generate_batch(const rocrand_b200_request* requests,
                                                      size_t                      count,
                                                      hipStream_t                 stream);

/* A batch laid out once and run many times (the same requests, e.g. a steady shape).
 * create: validates and uploads the descriptor table on `stream` (Poisson tables too);
 * execute: runs it on `stream`, asynchronously; with use_graph != 0 the first execute
 * captures the launch into a CUDA graph and later ones replay it;
 * destroy: waits for the device, then frees the plan. */
typedef struct rocrand_b200_batch_plan_st* rocrand_b200_batch_plan;
rocrand_status ROCRANDAPI rocrand_b200_create_batch_plan(rocrand_b200_batch_plan*    plan,
                                                         const rocrand_b200_request* requests,
                                                         size_t                      count,
                                                         hipStream_t                 stream);
rocrand_status ROCRANDAPI rocrand_b200_execute_batch_plan(rocrand_b200_batch_plan plan,
                                                          int                     use_graph,
                                                          hipStream_t             stream);
rocrand_status ROCRANDAPI rocrand_b200_destroy_batch_plan(rocrand_b200_batch_plan plan);

/* Chooses the batch kernel's tile size for every (generator, distribution) pair on the
 * current device by timing candidates on synthetic batches (allocates ~256 MiB of
 * scratch while it runs).  Later batches on any device use the chosen sizes. */
rocrand_status ROCRANDAPI rocrand_b200_autotune_batch(hipStream_t stream);

/* Reads the tile size in use for (rng_type, distribution), in output vectors (Philox),
 * engine slots (XORWOW, MRG32k3a) or points (Sobol32). */
rocrand_status ROCRANDAPI rocrand_b200_get_batch_tile(rocrand_rng_type          rng_type,
                                                      rocrand_b200_distribution distribution,
                                                      unsigned int*             units);

/*
 * Serving loop.  No counterpart in the reference.
 *
 * A server owns generator handles whose states stay resident on the device, an output pool
 * of `output_budget` bytes (allocated once), `streams` CUDA streams and a worker thread.
 * Requests queue in arrival order; the worker admits them as output memory frees up, packs
 * the admitted ones into one batched launch (continuous batching: up to `streams` batches
 * in flight, new arrivals join the next one) and completes them in any order.  Every
 * result equals the same sequence of calls made alone on a generator of the handle's type
 * and seed.  With plain_calls != 0 the server instead issues one ordinary generate call
 * per request on one stream (the per-request baseline, same admission and pool).
 * Handles: PHILOX4_32_10, XORWOW (or DEFAULT), MRG32K3A, QUASI_SOBOL32 (one dimension).
 */
typedef struct rocrand_b200_server_st* rocrand_b200_server;

rocrand_status ROCRANDAPI rocrand_b200_server_create(rocrand_b200_server* server,
                                                     size_t               output_budget,
                                                     unsigned int         streams,
                                                     int                  plain_calls);
/* Finishes the queued work, then frees the server, its handles and its pool. */
rocrand_status ROCRANDAPI rocrand_b200_server_destroy(rocrand_b200_server server);
/* Creates a generator (seeded now, on the device) and returns its handle. */
rocrand_status ROCRANDAPI rocrand_b200_server_add_generator(rocrand_b200_server server,
                                                            rocrand_rng_type    rng_type,
                                                            unsigned long long  seed,
                                                            unsigned int*       handle);
/* Queues n values of `distribution` (parameters as in rocrand_b200_request) from the
 * handle's generator; the output is allocated from the pool when the request is admitted.
 * ROCRAND_STATUS_OUT_OF_RANGE for n == 0 or an output larger than the budget (counted in
 * the pool's 512-byte granules); ROCRAND_STATUS_NOT_CREATED for an unknown handle. */
rocrand_status ROCRANDAPI rocrand_b200_server_submit(rocrand_b200_server       server,
                                                     unsigned int              handle,
                                                     rocrand_b200_distribution distribution,
                                                     double                    param0,
                                                     double                    param1,
                                                     size_t                    n,
                                                     unsigned long long*       ticket);
/* Blocks until the request is complete; returns its output (device memory, valid until
 * release) and its submit-to-complete latency. */
rocrand_status ROCRANDAPI rocrand_b200_server_wait(rocrand_b200_server server,
                                                   unsigned long long  ticket,
                                                   void**              output,
                                                   double*             latency_seconds);
/* Returns a completed request's output memory to the pool. */
rocrand_status ROCRANDAPI rocrand_b200_server_release(rocrand_b200_server server,
                                                      unsigned long long  ticket);

/* One request of a timed trace: submitted `arrival_seconds` after the trace starts. */
typedef struct rocrand_b200_trace_item
{
    double                    arrival_seconds;
    unsigned int              handle;
    rocrand_b200_distribution distribution;
    double                    param0;
    double                    param1;
    size_t                    n;
} rocrand_b200_trace_item;

/* Replays a trace in real time (outputs are released as they complete) and returns each
 * request's submit-to-complete latency and the wall time from start to the last completion. */
rocrand_status ROCRANDAPI rocrand_b200_server_run_trace(rocrand_b200_server            server,
                                                        const rocrand_b200_trace_item* items,
                                                        size_t                         count,
                                                        double*                        latency_seconds,
                                                        double*                        wall_seconds);

#if defined(__cplusplus)
}
#endif

#endif /* ROCRAND_B200_H_ */
