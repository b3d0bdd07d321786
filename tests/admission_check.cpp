// Host check of the serving loop's admission policy (rocrand_b200/csrc/admission.hpp):
// random queues of requests on stateful and stateless handles, random batch limits and
// output budgets; every admission must take exactly the requests, in the same order, that a
// plain scan of the whole queue takes, and leave the same queue behind.  Prints "ok <rounds>".
#include "../rocrand_b200/csrc/admission.hpp"

#include <algorithm>
#include <cstdio>
#include <deque>
#include <random>
#include <vector>

namespace
{

struct Req
{
    int      id;
    uint32_t handle;
    size_t   bytes;
};

// The policy written as a scan of the whole queue, with linear membership tests.
void admit_plain(std::deque<Req*>& q, std::vector<Req*>& out, size_t max_reqs, size_t max_bytes,
                 const std::vector<bool>& stateful, size_t& budget)
{
    std::vector<uint32_t> used, blocked;
    size_t                taken = 0;
    auto has = [](const std::vector<uint32_t>& v, uint32_t x) { return std::find(v.begin(), v.end(), x) != v.end(); };
    auto it  = q.begin();
    while(it != q.end() && out.size() < max_reqs)
    {
        Req* r = *it;
        if(has(blocked, r->handle) || (stateful[r->handle] && has(used, r->handle)))
        {
            if(!has(blocked, r->handle))
                blocked.push_back(r->handle);
            ++it;
            continue;
        }
        if(!out.empty() && taken + r->bytes > max_bytes)
            break;
        if(r->bytes > budget)
            break;
        budget -= r->bytes;
        taken += r->bytes;
        if(stateful[r->handle])
            used.push_back(r->handle);
        out.push_back(r);
        it = q.erase(it);
    }
}

} // namespace

int main()
{
    std::mt19937_64 rng(12345);
    int             rounds = 0;
    for(int trial = 0; trial < 400; trial++)
    {
        const uint32_t    handles = 1 + rng() % 70;
        std::vector<bool> stateful(handles);
        const int         mode = trial % 3; // all stateful, all stateless, mixed
        for(uint32_t h = 0; h < handles; h++)
            stateful[h] = mode == 0 ? true : mode == 1 ? false : (rng() & 1) != 0;
        std::deque<Req>             store;
        std::deque<Req*>            plain_q;
        rb200::AdmissionQueue<Req>  q;
        size_t                      budget_a = 0, budget_b = 0;
        int                         next_id  = 0;
        for(int step = 0; step < 120; step++)
        {
            const int pushes = static_cast<int>(rng() % (step == 0 ? 400 : 40));
            for(int k = 0; k < pushes; k++)
            {
                // skewed handle choice, so some handles pile up long runs of requests
                const uint32_t h = static_cast<uint32_t>(rng() % 4 == 0 ? rng() % std::min<uint32_t>(handles, 3)
                                                                        : rng() % handles);
                store.push_back(Req{next_id++, h, 1 + rng() % 1000});
                plain_q.push_back(&store.back());
                q.push(&store.back(), h);
            }
            const size_t add = rng() % 20000;
            budget_a += add;
            budget_b += add;
            const size_t max_reqs  = rng() % 4 == 0 ? 1 : 1 + rng() % 64;
            const size_t max_bytes = rng() % 3 == 0 ? size_t(1) << 40 : 1 + rng() % 30000;
            std::vector<Req*> out_a, out_b;
            admit_plain(plain_q, out_a, max_reqs, max_bytes, stateful, budget_a);
            q.admit(
                out_b, max_reqs, max_bytes, [&](const Req* r) { return static_cast<bool>(stateful[r->handle]); },
                [](const Req* r) { return r->bytes; },
                [&](Req* r) {
                    if(r->bytes > budget_b)
                        return false;
                    budget_b -= r->bytes;
                    return true;
                });
            if(out_a != out_b || budget_a != budget_b)
            {
                std::printf("mismatch: trial %d step %d admitted %zu vs %zu\n", trial, step, out_a.size(), out_b.size());
                return 1;
            }
            std::vector<Req*> rest;
            q.for_each([&](Req* r) { rest.push_back(r); });
            if(rest != std::vector<Req*>(plain_q.begin(), plain_q.end()) || q.size() != plain_q.size())
            {
                std::printf("queue differs: trial %d step %d\n", trial, step);
                return 1;
            }
            // finished requests give their memory back
            for(Req* r : out_a)
                if(rng() % 2)
                {
                    budget_a += r->bytes;
                    budget_b += r->bytes;
                }
            rounds++;
        }
    }
    std::printf("ok %d\n", rounds);
    return 0;
}
