// host_exec.hpp -- running a generate call's output positions on the host's cores (the CPU
// path of host generators).  Every output position is a pure function of the engine
// position and the call, as in the kernels, so disjoint ranges can run on separate threads
// and give the same bytes as one thread.
#pragma once

#include <algorithm>
#include <thread>
#include <vector>

namespace rb200
{

// f(begin, end) over [0, n) in contiguous chunks, one per host thread (one chunk when n is
// below `grain`: positions cheap enough that threads would cost more than they save).
template<class F>
void host_parallel_for(unsigned long long n, F&& f, unsigned long long grain = 1ull << 15)
{
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if(n < grain || hw == 1)
    {
        f(0ull, n);
        return;
    }
    const unsigned long long chunk = (n + hw - 1) / hw;
    std::vector<std::thread> pool;
    for(unsigned t = 0; t < hw; t++)
    {
        const unsigned long long b = t * chunk;
        const unsigned long long e = std::min(n, b + chunk);
        if(b >= e)
            break;
        pool.emplace_back([&f, b, e] { f(b, e); });
    }
    for(auto& th : pool)
        th.join();
}

} // namespace rb200
