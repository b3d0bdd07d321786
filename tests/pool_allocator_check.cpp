// Host check of the serving loop's output-pool allocator (rocrand_b200/csrc/pool_allocator.hpp):
// random allocations and releases against a list of the live ranges.  Every allocation must
// lie inside the pool, overlap no live range, start at the lowest offset where its granules
// fit (first fit), and fail only when no such offset exists; the free list must stay ordered,
// coalesced and equal to the complement of the live ranges.  Prints "ok <operations>".
#include "../rocrand_b200/csrc/pool_allocator.hpp"

#include <algorithm>
#include <cstdio>
#include <random>
#include <utility>
#include <vector>

namespace
{

using Range = std::pair<size_t, size_t>; // offset, granule bytes

// Lowest offset where `bytes` fit between the live ranges, or SIZE_MAX.
size_t first_fit(std::vector<Range> live, size_t bytes, size_t budget)
{
    std::sort(live.begin(), live.end());
    size_t at = 0;
    for(const Range& r : live)
    {
        if(r.first >= at + bytes)
            return at;
        at = std::max(at, r.first + r.second);
    }
    return at + bytes <= budget ? at : SIZE_MAX;
}

bool free_list_matches(const rb200::PoolAllocator& a, std::vector<Range> live, size_t budget)
{
    std::sort(live.begin(), live.end());
    std::vector<Range> gaps;
    size_t             at = 0;
    for(const Range& r : live)
    {
        if(r.first > at)
            gaps.push_back({at, r.first - at});
        at = r.first + r.second;
    }
    if(budget > at)
        gaps.push_back({at, budget - at});
    std::vector<Range> got(a.free_ranges().begin(), a.free_ranges().end());
    return got == gaps;
}

} // namespace

int main()
{
    std::mt19937_64 rng(777);
    long            ops = 0;
    for(int trial = 0; trial < 300; trial++)
    {
        // budgets in and out of granule multiples
        const size_t budget = (1 + rng() % 400) * 512 + (trial % 3 == 0 ? rng() % 512 : 0);
        rb200::PoolAllocator a;
        a.reset(budget);
        std::vector<Range> live;
        for(int step = 0; step < 400; step++, ops++)
        {
            if(live.empty() || rng() % 3 != 0)
            {
                const size_t bytes = 1 + rng() % (rng() % 4 == 0 ? budget : budget / 8 + 1);
                const size_t want  = first_fit(live, rb200::PoolAllocator::granules(bytes), budget);
                size_t       off   = 0;
                const bool   ok    = a.alloc(bytes, off);
                if(ok != (want != SIZE_MAX) || (ok && off != want))
                {
                    std::printf("alloc differs: trial %d step %d ok %d off %zu want %zu\n", trial, step, ok, off, want);
                    return 1;
                }
                if(ok)
                    live.push_back({off, rb200::PoolAllocator::granules(bytes)});
            }
            else
            {
                const size_t k = rng() % live.size();
                // release with the request's byte count (any count that rounds to the same granules)
                a.release(live[k].first, live[k].second - rng() % 512);
                live.erase(live.begin() + static_cast<long>(k));
            }
            size_t used = 0;
            for(const Range& r : live)
                used += r.second;
            if(a.used() != used || !free_list_matches(a, live, budget))
            {
                std::printf("free list differs: trial %d step %d\n", trial, step);
                return 1;
            }
        }
        while(!live.empty())
        {
            a.release(live.back().first, live.back().second);
            live.pop_back();
        }
        if(a.used() != 0 || a.free_ranges().size() != 1 || a.free_ranges().begin()->second != budget)
        {
            std::printf("not coalesced after releasing everything: trial %d\n", trial);
            return 1;
        }
    }
    std::printf("ok %ld\n", ops);
    return 0;
}
