// pool_allocator.hpp -- first-fit allocator over the serving loop's output pool (no CUDA,
// so host tests run it).
//
// Offsets into one pre-allocated pool, in 512-byte granules: allocation takes the free range
// with the lowest offset that is large enough, release returns a range and merges it with
// free neighbours, so the free list stays coalesced and ordered by offset.
#pragma once

#include <cstddef>
#include <iterator>
#include <map>

namespace rb200
{

class PoolAllocator
{
public:
    static constexpr size_t kGranule = 512;
    static size_t granules(size_t bytes) { return (bytes + kGranule - 1) & ~(kGranule - 1); }

    void reset(size_t bytes)
    {
        m_free.clear();
        m_free[0] = bytes;
        m_used    = 0;
    }
    bool alloc(size_t bytes, size_t& off)
    {
        bytes = granules(bytes);
        for(auto it = m_free.begin(); it != m_free.end(); ++it)
        {
            if(it->second < bytes)
                continue;
            off              = it->first;
            const size_t rem = it->second - bytes;
            m_free.erase(it);
            if(rem)
                m_free[off + bytes] = rem;
            m_used += bytes;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes)
    {
        bytes = granules(bytes);
        m_used -= bytes;
        auto next = m_free.lower_bound(off);
        if(next != m_free.end() && off + bytes == next->first)
        {
            bytes += next->second;
            next = m_free.erase(next);
        }
        if(next != m_free.begin())
        {
            auto prev = std::prev(next);
            if(prev->first + prev->second == off)
            {
                prev->second += bytes;
                return;
            }
        }
        m_free[off] = bytes;
    }
    size_t used() const { return m_used; }
    // Free ranges (offset -> size) in offset order.
    const std::map<size_t, size_t>& free_ranges() const { return m_free; }

private:
    std::map<size_t, size_t> m_free;
    size_t                   m_used = 0;
};

} // namespace rb200
