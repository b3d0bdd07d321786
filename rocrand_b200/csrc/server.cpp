// server.cpp -- serving loop: continuous batching of generate requests on resident
// generator states.
//
// A server owns generator handles (states resident on the device for their lifetime), an
// output pool of a fixed budget, and a worker thread.  Requests are queued by submit();
// the worker admits them in arrival order as output memory frees up, packs the admitted
// ones into one batch (batch.hpp: one persistent launch over a descriptor table), and keeps
// up to `streams` batches in flight, so requests arriving while others run start as soon
// as a stream and memory are free.  A stateful handle (XORWOW, MRG32k3a) is in at most one
// batch at a time and its next batch waits on the previous one's event; Philox and Sobol
// handles keep their position on the host and may appear several times in one batch.
// Each result equals the same call made alone on the handle's generator: descriptors are
// taken in submission order from the generator's own state (batch_descriptor).
// Requests of at least kDirectBytes run as their own ordinary call on a separate stream as
// soon as they are admitted: at that size the call streams at the kernel's own speed, and
// outside a batch it does not hold back the small requests it was admitted with (a batch
// completes as a whole).  A request that finds no other queued runs alone as an ordinary
// call on a third stream, so batching costs a lone request no waiting.  Poisson requests go
// through batches (whose tables are shared per lambda across streams) or, alone, through
// the single-request stream.
// The plain mode runs the same admission and memory pool but issues one ordinary
// generate call per request on one stream: the per-request baseline.
#include "admission.hpp"
#include "batch.hpp"
#include "common.hpp"
#include "generators.hpp"
#include "pool_allocator.hpp"

#include <rocrand_b200.h>

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace rb200
{
namespace
{

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Handle;

struct Request
{
    unsigned long long ticket;
    uint32_t           handle;
    Handle*            h = nullptr; // stable: handles live in a deque
    uint32_t           dist;
    double             p0, p1;
    size_t             n, bytes;
    size_t             off   = 0;
    int                state = 0; // 0 queued, 1 in flight, 2 done, 3 failed
    rocrand_status     status = ROCRAND_STATUS_SUCCESS;
    double             t_submit = 0, t_done = 0;
    bool               release_when_done = false;
};

struct Handle
{
    std::unique_ptr<rocrand_generator_base_type> gen;
    bool                                         stateful    = false;
    cudaEvent_t                                  last        = nullptr; // its last batch
    bool                                         last_pending = false;
};

struct InFlight
{
    cudaEvent_t           done = nullptr;
    int                   stream = 0;
    std::vector<Request*> reqs;
};

} // namespace

class Server
{
public:
    Server(size_t budget, unsigned streams, int plain) : m_budget(budget), m_plain(plain != 0)
    {
        m_nstreams = plain ? 1u : std::max(1u, std::min(streams, 8u));
    }

    rocrand_status start()
    {
        if(cudaGetDevice(&m_device) != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        if(cudaMalloc(&m_pool, m_budget) != cudaSuccess)
        {
            m_pool = nullptr;
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        }
        m_alloc.reset(m_budget);
        for(unsigned s = 0; s < m_nstreams; s++)
        {
            cudaStream_t st = nullptr;
            if(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
                return ROCRAND_STATUS_INTERNAL_ERROR;
            m_streams.push_back(st);
            m_plans.emplace_back(new BatchPlan());
            m_plans.back()->set_serving(true);
            // tables for a large batch now, not on the request path (allocation is slow and
            // freeing a table to grow it waits for the whole device)
            const rocrand_status rst
                = m_plain ? ROCRAND_STATUS_SUCCESS : m_plans.back()->reserve(kMaxBatchRequests, size_t(1) << 20);
            if(rst != ROCRAND_STATUS_SUCCESS)
                return rst;
        }
        if(!m_plain
           && (cudaStreamCreateWithFlags(&m_direct, cudaStreamNonBlocking) != cudaSuccess
               || cudaStreamCreateWithFlags(&m_single, cudaStreamNonBlocking) != cudaSuccess))
            return ROCRAND_STATUS_INTERNAL_ERROR;
        m_worker = std::thread([this] { loop(); });
        return ROCRAND_STATUS_SUCCESS;
    }

    ~Server()
    {
        {
            std::lock_guard<std::mutex> lock(m_mu);
            m_stop = true;
        }
        m_cv.notify_all();
        if(m_worker.joinable())
            m_worker.join();
        cudaSetDevice(m_device);
        for(auto s : m_streams)
            cudaStreamSynchronize(s);
        if(m_direct)
            cudaStreamSynchronize(m_direct);
        if(m_single)
            cudaStreamSynchronize(m_single);
        m_plans.clear();
        for(auto s : m_streams)
            cudaStreamDestroy(s);
        if(m_direct)
            cudaStreamDestroy(m_direct);
        if(m_single)
            cudaStreamDestroy(m_single);
        for(auto& h : m_handles)
            if(h.last)
                cudaEventDestroy(h.last);
        m_handles.clear();
        cudaFree(m_pool);
    }

    rocrand_status add_generator(rocrand_rng_type type, unsigned long long seed, uint32_t& id)
    {
        std::unique_ptr<rocrand_generator_base_type> g(make_generator(type));
        if(!g)
            return ROCRAND_STATUS_TYPE_ERROR;
        const bool stateful = type == ROCRAND_RNG_PSEUDO_XORWOW || type == ROCRAND_RNG_PSEUDO_DEFAULT
                              || type == ROCRAND_RNG_PSEUDO_MRG32K3A;
        const bool ok = stateful || type == ROCRAND_RNG_PSEUDO_PHILOX4_32_10
                        || type == ROCRAND_RNG_QUASI_SOBOL32 || type == ROCRAND_RNG_QUASI_DEFAULT;
        if(!ok)
            return ROCRAND_STATUS_TYPE_ERROR;
        rocrand_status st = g->set_seed(seed);
        if(st == ROCRAND_STATUS_SUCCESS)
            st = g->set_stream(m_streams[0]);
        if(st == ROCRAND_STATUS_SUCCESS)
            st = g->init(); // the resident state is seeded now, on the server's stream
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        if(cudaStreamSynchronize(m_streams[0]) != cudaSuccess)
            return ROCRAND_STATUS_LAUNCH_FAILURE;
        Handle h;
        h.gen      = std::move(g);
        h.stateful = stateful;
        if(cudaEventCreateWithFlags(&h.last, cudaEventDisableTiming) != cudaSuccess)
            return ROCRAND_STATUS_INTERNAL_ERROR;
        std::lock_guard<std::mutex> lock(m_mu);
        id = static_cast<uint32_t>(m_handles.size());
        m_handles.push_back(std::move(h));
        return ROCRAND_STATUS_SUCCESS;
    }

    // t_arrival: when the request arrived (steady clock seconds), 0 = now; latency is
    // measured from it, so time a late submitter spends is queueing latency too.
    rocrand_status submit(uint32_t handle, uint32_t dist, double p0, double p1, size_t n,
                          bool release_when_done, double t_arrival, unsigned long long& ticket)
    {
        if(dist >= BD_COUNT)
            return ROCRAND_STATUS_TYPE_ERROR;
        if(n == 0)
            return ROCRAND_STATUS_OUT_OF_RANGE;
        if(n > m_budget / batch_elem_size(dist)) // also keeps n * element size from wrapping
            return ROCRAND_STATUS_OUT_OF_RANGE;
        const size_t bytes = n * batch_elem_size(dist);
        // the pool hands out whole granules: a request whose granules exceed the budget could
        // never be admitted, and admission does not overtake
        if(PoolAllocator::granules(bytes) > m_budget)
            return ROCRAND_STATUS_OUT_OF_RANGE;
        std::lock_guard<std::mutex> lock(m_mu);
        if(handle >= m_handles.size())
            return ROCRAND_STATUS_NOT_CREATED;
        auto r               = std::make_unique<Request>();
        r->ticket            = ++m_next_ticket;
        r->handle            = handle;
        r->h                 = &m_handles[handle];
        r->dist              = dist;
        r->p0                = p0;
        r->p1                = p1;
        r->n                 = n;
        r->bytes             = bytes;
        r->t_submit          = t_arrival > 0 ? t_arrival : now_s();
        r->release_when_done = release_when_done;
        ticket               = r->ticket;
        m_queue.push(r.get(), handle);
        m_reqs[ticket] = std::move(r);
        m_cv.notify_all();
        return ROCRAND_STATUS_SUCCESS;
    }

    rocrand_status wait(unsigned long long ticket, void** out, double* latency)
    {
        std::unique_lock<std::mutex> lock(m_mu);
        auto                         it = m_reqs.find(ticket);
        if(it == m_reqs.end())
            return ROCRAND_STATUS_OUT_OF_RANGE;
        Request* r = it->second.get();
        m_done_cv.wait(lock, [&] { return r->state >= 2; });
        if(out)
            *out = r->release_when_done ? nullptr : m_pool + r->off;
        if(latency)
            *latency = r->t_done - r->t_submit;
        return r->status;
    }

    rocrand_status release(unsigned long long ticket)
    {
        std::lock_guard<std::mutex> lock(m_mu);
        auto                        it = m_reqs.find(ticket);
        if(it == m_reqs.end())
            return ROCRAND_STATUS_OUT_OF_RANGE;
        Request* r = it->second.get();
        if(r->state < 2)
            return ROCRAND_STATUS_OUT_OF_RANGE; // still running
        if(!r->release_when_done && r->state == 2)
            m_alloc.release(r->off, r->bytes);
        m_reqs.erase(it);
        m_cv.notify_all();
        return ROCRAND_STATUS_SUCCESS;
    }

private:
    // Takes queued requests in arrival order while output memory lasts (admission.hpp: a
    // request that does not fit stops admission, a stateful handle joins a batch once).
    void admit(std::vector<Request*>& out, size_t max_reqs, size_t max_bytes)
    {
        m_queue.admit(
            out, max_reqs, max_bytes, [](const Request* r) { return r->h->stateful; },
            [](const Request* r) { return r->bytes; },
            [this](Request* r) {
                size_t off = 0;
                if(!m_alloc.alloc(r->bytes, off))
                    return false;
                r->off   = off;
                r->state = 1;
                return true;
            });
    }

    void finish(Request* r, rocrand_status st)
    {
        r->status = st;
        r->t_done = now_s();
        r->state  = st == ROCRAND_STATUS_SUCCESS ? 2 : 3;
        if(r->release_when_done || st != ROCRAND_STATUS_SUCCESS)
            m_alloc.release(r->off, r->bytes);
        if(r->release_when_done && st == ROCRAND_STATUS_SUCCESS)
        {
            // kept only for its latency until wait/release
        }
    }

    // One ordinary generate call for a request on `stream`.
    rocrand_status plain_call(Request* r, cudaStream_t stream)
    {
        Handle& h = *r->h;
        h.gen->set_stream(stream);
        void*          out = m_pool + r->off;
        rocrand_status st;
        DistParams     dp;
        switch(r->dist)
        {
            case BD_UINT: st = h.gen->generate(out, r->n, Dist::U32, dp); break;
            case BD_FLOAT: st = h.gen->generate(out, r->n, Dist::F32, dp); break;
            case BD_DOUBLE: st = h.gen->generate(out, r->n, Dist::F64, dp); break;
            case BD_NORMAL_F:
                dp.mean_f = static_cast<float>(r->p0);
                dp.std_f  = static_cast<float>(r->p1);
                st        = h.gen->generate(out, r->n, Dist::NORMAL_F32, dp);
                break;
            default: st = h.gen->generate_poisson(static_cast<unsigned int*>(out), r->n, r->p0); break;
        }
        return st;
    }

    // Launches one batch (or, in plain mode, one ordinary call) of admitted requests.
    rocrand_status launch(std::vector<Request*>& reqs, int s)
    {
        cudaStream_t stream = m_streams[s];
        if(m_plain)
        {
            return plain_call(reqs[0], stream);
        }
        // each stream reuses its own descriptor table: its previous batch is finished
        BatchPlan& plan = *m_plans[s];
        plan.clear();
        for(Request* r : reqs)
        {
            Handle&  h = *r->h;
            BatchReq d;
            rocrand_status st
                = h.gen->batch_descriptor(r->dist, r->p0, r->p1, m_pool + r->off, r->n, d, stream);
            if(st != ROCRAND_STATUS_SUCCESS)
                return st;
            plan.add(d);
            if(h.stateful && h.last_pending)
                cudaStreamWaitEvent(stream, h.last, 0);
        }
        rocrand_status st = plan.upload(stream);
        if(st == ROCRAND_STATUS_SUCCESS)
            st = plan.launch(stream);
        return st;
    }

    // A request as its own ordinary call on `stream` (the direct or the single-request
    // stream), after its handle's previous batch or call (stateful handles); records the
    // handle's last event.  Poisson requests come here only on the single-request stream,
    // so a generator's own Poisson table is only ever refreshed and read there.
    rocrand_status launch_alone(Request* r, cudaStream_t stream)
    {
        Handle& h = *r->h;
        if(h.stateful && h.last_pending)
            cudaStreamWaitEvent(stream, h.last, 0);
        const rocrand_status st = plain_call(r, stream);
        if(st == ROCRAND_STATUS_SUCCESS && h.stateful)
        {
            cudaEventRecord(h.last, stream);
            h.last_pending = true;
        }
        return st;
    }

    void loop()
    {
        cudaSetDevice(m_device);
        std::deque<InFlight> inflight;
        std::vector<bool>    busy(m_nstreams, false);
        std::unique_lock<std::mutex> lock(m_mu);
        for(;;)
        {
            // retire finished batches
            bool retired = false;
            for(auto it = inflight.begin(); it != inflight.end();)
            {
                if(cudaEventQuery(it->done) != cudaSuccess)
                {
                    ++it;
                    continue;
                }
                for(Request* r : it->reqs)
                    finish(r, ROCRAND_STATUS_SUCCESS);
                if(it->stream >= 0)
                    busy[it->stream] = false;
                else if(it->stream == kSingleStream)
                    m_singles--;
                cudaEventDestroy(it->done);
                it      = inflight.erase(it);
                retired = true;
            }
            if(retired)
            {
                for(auto& h : m_handles)
                    if(h.last_pending && cudaEventQuery(h.last) == cudaSuccess)
                        h.last_pending = false;
                m_done_cv.notify_all();
            }
            if(m_stop && m_queue.empty() && inflight.empty())
                return;
            // What to start:
            //  * plain mode: one ordinary call per request on stream 0, queued back to back;
            //  * otherwise, with kMinBatchQueue or more requests queued and a batch stream
            //    free: a batch of what admission takes; with fewer queued (or every batch
            //    stream busy): the oldest request alone as an ordinary call on the
            //    single-request stream, so a short queue is served exactly as plain calls
            //    (a batch's plan upload costs more than it saves for two or three small
            //    requests) and no request waits for others to gather or for a batch stream.
            //  In both, admitted requests of at least kDirectBytes run as ordinary calls on
            //  the direct stream.
            int  s     = -1;
            bool batch = false;
            if(m_plain)
                s = inflight.size() < kPlainInFlight ? 0 : -1;
            else
            {
                for(unsigned k = 0; k < m_nstreams; k++)
                    if(!busy[k])
                    {
                        s = static_cast<int>(k);
                        break;
                    }
                batch = s >= 0 && m_queue.size() >= kMinBatchQueue;
            }
            const bool single = !m_plain && !batch && m_singles < kPlainInFlight;
            if(!m_queue.empty() && (m_plain ? s >= 0 : (batch || single)))
            {
                std::vector<Request*> reqs;
                admit(reqs, batch ? kMaxBatchRequests : 1, m_plain ? m_budget : (size_t(8) << 30));
                // large requests: their own ordinary call on the direct stream; a batch that
                // keeps one request runs it as a single
                std::vector<Request*> direct, singles;
                if(!m_plain)
                {
                    size_t k = 0;
                    for(size_t i = 0; i < reqs.size(); i++)
                    {
                        Request* r = reqs[i];
                        if(r->bytes >= kDirectBytes && r->dist != BD_POISSON)
                            direct.push_back(r);
                        else
                            reqs[k++] = r;
                    }
                    reqs.resize(k);
                    if(reqs.size() == 1)
                    {
                        singles.push_back(reqs[0]);
                        reqs.clear();
                    }
                }
                if(!reqs.empty() || !direct.empty() || !singles.empty())
                {
                    // admitted requests, their handles and the streams belong to this thread:
                    // launch without holding the queue lock, so submitters are not delayed
                    lock.unlock();
                    std::vector<std::pair<Request*, rocrand_status>> own_st;
                    for(Request* r : direct)
                        own_st.emplace_back(r, launch_alone(r, m_direct));
                    const size_t n_direct = own_st.size();
                    for(Request* r : singles)
                        own_st.emplace_back(r, launch_alone(r, m_single));
                    rocrand_status st = reqs.empty() ? ROCRAND_STATUS_SUCCESS : launch(reqs, s);
                    lock.lock();
                    for(size_t i = 0; i < own_st.size(); i++)
                    {
                        Request* const       r   = own_st[i].first;
                        const rocrand_status rst = own_st[i].second;
                        if(rst != ROCRAND_STATUS_SUCCESS)
                        {
                            finish(r, rst);
                            continue;
                        }
                        InFlight f;
                        f.stream = i < n_direct ? kDirectStream : kSingleStream;
                        cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming);
                        cudaEventRecord(f.done, i < n_direct ? m_direct : m_single);
                        f.reqs.push_back(r);
                        if(i >= n_direct)
                            m_singles++;
                        inflight.push_back(std::move(f));
                    }
                    if(!own_st.empty())
                        m_done_cv.notify_all();
                    if(reqs.empty())
                        continue;
                    InFlight f;
                    f.stream = s;
                    if(st != ROCRAND_STATUS_SUCCESS)
                    {
                        for(Request* r : reqs)
                            finish(r, st);
                        m_done_cv.notify_all();
                        continue;
                    }
                    cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming);
                    cudaEventRecord(f.done, m_streams[s]);
                    if(!m_plain)
                        for(Request* r : reqs)
                        {
                            Handle& h = *r->h;
                            if(h.stateful)
                            {
                                cudaEventRecord(h.last, m_streams[s]);
                                h.last_pending = true;
                            }
                        }
                    f.reqs = std::move(reqs);
                    busy[s] = !m_plain;
                    inflight.push_back(std::move(f));
                    continue;
                }
            }
            // nothing to start: poll the device again shortly, or sleep until a submit
            if(inflight.empty())
                m_cv.wait_for(lock, std::chrono::milliseconds(2));
            else
            {
                lock.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(5));
                lock.lock();
            }
        }
    }

    static constexpr size_t       kMaxBatchRequests = 8192;
    static constexpr size_t       kMinBatchQueue    = 4;
    static constexpr size_t       kPlainInFlight  = 4096;
    static constexpr size_t       kDirectBytes    = size_t(32) << 20;
    static constexpr int          kDirectStream   = -1; // InFlight::stream of a direct call
    static constexpr int          kSingleStream   = -2; // ... and of a single request
    size_t                        m_budget;
    bool                          m_plain;
    unsigned                      m_nstreams = 1;
    int                           m_device   = 0;
    unsigned char*                m_pool     = nullptr;
    PoolAllocator                 m_alloc;
    std::vector<cudaStream_t>     m_streams;
    cudaStream_t                  m_direct = nullptr; // large requests as ordinary calls
    cudaStream_t                  m_single = nullptr; // lone requests as ordinary calls
    size_t                        m_singles = 0;      // single-request calls in flight
    std::vector<std::unique_ptr<BatchPlan>> m_plans;
    std::deque<Handle>            m_handles;
    AdmissionQueue<Request>       m_queue;
    std::unordered_map<unsigned long long, std::unique_ptr<Request>> m_reqs;
    unsigned long long            m_next_ticket = 0;
    std::mutex                    m_mu;
    std::condition_variable       m_cv, m_done_cv;
    std::thread                   m_worker;
    bool                          m_stop        = false;
};

} // namespace rb200

using namespace rb200;

struct rocrand_b200_server_st
{
    std::unique_ptr<Server> s;
};

extern "C" rocrand_status ROCRANDAPI rocrand_b200_server_create(rocrand_b200_server* server,
                                                                size_t output_budget,
                                                                unsigned int streams, int plain_calls)
{
    if(server == nullptr || output_budget == 0)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        auto h = std::make_unique<rocrand_b200_server_st>();
        h->s.reset(new Server(output_budget, streams, plain_calls));
        const rocrand_status st = h->s->start();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        *server = h.release();
        return ROCRAND_STATUS_SUCCESS;
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_server_destroy(rocrand_b200_server server)
{
    if(server == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    delete server;
    return ROCRAND_STATUS_SUCCESS;
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_server_add_generator(rocrand_b200_server server,
                                                                       rocrand_rng_type    rng_type,
                                                                       unsigned long long  seed,
                                                                       unsigned int*       handle)
{
    if(server == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    if(handle == nullptr)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        uint32_t             id = 0;
        const rocrand_status st = server->s->add_generator(rng_type, seed, id);
        *handle                 = id;
        return st;
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_server_submit(rocrand_b200_server       server,
                                                                unsigned int              handle,
                                                                rocrand_b200_distribution distribution,
                                                                double param0, double param1,
                                                                size_t n, unsigned long long* ticket)
{
    if(server == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    if(ticket == nullptr)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        return server->s->submit(handle, static_cast<uint32_t>(distribution), param0, param1, n,
                                 false, 0.0, *ticket);
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_server_wait(rocrand_b200_server server,
                                                              unsigned long long ticket, void** output,
                                                              double* latency_seconds)
{
    if(server == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    try
    {
        return server->s->wait(ticket, output, latency_seconds);
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_server_release(rocrand_b200_server server,
                                                                 unsigned long long  ticket)
{
    if(server == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    try
    {
        return server->s->release(ticket);
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}

extern "C" rocrand_status ROCRANDAPI rocrand_b200_server_run_trace(rocrand_b200_server server,
                                                                   const rocrand_b200_trace_item* items,
                                                                   size_t count, double* latency_seconds,
                                                                   double* wall_seconds)
{
    if(server == nullptr)
        return ROCRAND_STATUS_NOT_CREATED;
    if(items == nullptr && count > 0)
        return ROCRAND_STATUS_OUT_OF_RANGE;
    try
    {
        std::vector<unsigned long long> tickets(count);
        const double                    t0 = now_s();
        for(size_t i = 0; i < count; i++)
        {
            const double due = t0 + items[i].arrival_seconds;
            while(now_s() < due)
            {
            }
            const rocrand_status st
                = server->s->submit(items[i].handle, static_cast<uint32_t>(items[i].distribution),
                                    items[i].param0, items[i].param1, items[i].n, true, due,
                                    tickets[i]);
            if(st != ROCRAND_STATUS_SUCCESS)
                return st;
        }
        for(size_t i = 0; i < count; i++)
        {
            double               lat = 0;
            const rocrand_status st  = server->s->wait(tickets[i], nullptr, &lat);
            if(st != ROCRAND_STATUS_SUCCESS)
                return st;
            if(latency_seconds)
                latency_seconds[i] = lat;
            server->s->release(tickets[i]);
        }
        // every request is complete once the last wait returns
        if(wall_seconds)
            *wall_seconds = now_s() - t0;
        return ROCRAND_STATUS_SUCCESS;
    }
    catch(...)
    {
        return ROCRAND_STATUS_INTERNAL_ERROR;
    }
}
