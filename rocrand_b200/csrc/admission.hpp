// admission.hpp -- the serving loop's admission policy (no CUDA, so host tests run it).
//
// Requests wait in arrival order.  A batch takes them in that order while output memory
// lasts; a request that does not fit stops admission (no overtaking).  A stateful handle
// (one resident engine state: XORWOW, MRG32k3a) joins a batch at most once, so its later
// requests, and anything after a skipped request of the same handle, wait for the next batch
// in their order, while other handles' requests go ahead of them.
//
// The queue is a list with per-handle counts and marks, so one admission costs the requests
// it visits, and the scan ends as soon as every request left belongs to a handle that is
// already blocked for this batch: with a backlog of one stateful handle's requests (a
// saturated trace) a batch no longer walks the whole queue.
#pragma once

#include <cstddef>
#include <cstdint>
#include <list>
#include <vector>

namespace rb200
{

template<class Req>
class AdmissionQueue
{
public:
    void push(Req* r, uint32_t handle)
    {
        if(handle >= m_queued.size())
        {
            m_queued.resize(handle + 1, 0);
            m_used.resize(handle + 1, 0);
            m_blocked.resize(handle + 1, 0);
        }
        m_q.push_back(Entry{r, handle});
        m_queued[handle]++;
    }

    size_t size() const { return m_q.size(); }
    bool   empty() const { return m_q.empty(); }

    // Appends the admitted requests to `out` (at most max_reqs; at most max_bytes unless the
    // first request alone is larger).  stateful(r): r's handle holds one state; bytes(r): r's
    // output size; reserve(r): takes r's output memory, false when it does not fit.
    template<class Stateful, class Bytes, class Reserve>
    void admit(std::vector<Req*>& out, size_t max_reqs, size_t max_bytes, Stateful stateful, Bytes bytes,
               Reserve reserve)
    {
        const size_t first = out.size();
        ++m_epoch;
        size_t remaining     = m_q.size(); // entries from `it` to the end
        size_t blocked_ahead = 0;          // of those, entries of blocked handles
        size_t taken         = 0;
        auto   it            = m_q.begin();
        while(it != m_q.end() && out.size() - first < max_reqs && blocked_ahead < remaining)
        {
            Req* const     r = it->req;
            const uint32_t h = it->handle;
            if(m_blocked[h] == m_epoch)
            {
                --blocked_ahead;
                --remaining;
                ++it;
                continue;
            }
            if(m_used[h] == m_epoch)
            {
                // a stateful handle's second request: it and all the handle's later ones wait
                // (its earlier requests were all admitted, so every queued one is ahead)
                m_blocked[h] = m_epoch;
                blocked_ahead += m_queued[h] - 1;
                --remaining;
                ++it;
                continue;
            }
            const size_t b = bytes(r);
            if(out.size() > first && taken + b > max_bytes)
                break;
            if(!reserve(r))
                break;
            taken += b;
            if(stateful(r))
                m_used[h] = m_epoch;
            out.push_back(r);
            m_queued[h]--;
            --remaining;
            it = m_q.erase(it);
        }
    }

    // Queued requests in order (for tests and diagnostics).
    template<class F>
    void for_each(F f) const
    {
        for(const Entry& e : m_q)
            f(e.req);
    }

private:
    struct Entry
    {
        Req*     req;
        uint32_t handle;
    };
    std::list<Entry>      m_q;
    std::vector<uint32_t> m_queued;  // per handle: its requests in the queue
    std::vector<uint64_t> m_used;    // per handle: epoch in which a stateful handle joined
    std::vector<uint64_t> m_blocked; // per handle: epoch in which it was blocked
    uint64_t              m_epoch = 0;
};

} // namespace rb200
