// Writes the table with which the kernels reproduce the host C library's logf on the
// arguments of the inverse-erf normal (logf_replay.cuh; reference rocrand_normal.h:174-194
// roc_f_erfinv, reached through normal_distribution(unsigned int), rocrand_normal.h:228-233).
//
//   make_logf_replay <out.bin>
//
// 1. Every argument the formula can reach: for each 32-bit Sobol value v (a 64-bit value
//    uses its high word), p = 2^-32 + v 2^-32 rounded once (uniform_distribution,
//    rocrand_uniform.h:61-64), x = 2p - 1, t = (1 - x)(1 + x), each operation rounded to
//    float as the kernels round it.
// 2. For each distinct t, the host's logf(t) against the kernels' float f of the logarithm
//    (logf_replay.cuh base(), compiled here for the host: the same IEEE operations).  Where
//    they differ, the host's result must be f's neighbour on the logarithm's side of f; the
//    argument joins the member set, and the bound of its bucket and side is raised to its
//    distance from the midpoint plus one.
// 3. The member set goes into a bucketed two-choice hash table (four keys per bucket, cuckoo
//    insertion; the table doubles until every key has a place).
// 4. Every t is replayed through logf_replay.cuh logf_host() with the finished tables and
//    must give the host's logf(t) bit for bit; otherwise nothing is written.
//
// Output (little-endian): "RBLOGF02", u32 bucket shift, u32 bucket count, u32 log2 of the
// key-bucket count, u32 members, u32 reachable arguments, u32 0; u32 bounds [bucket count]
// (side 0 in the low half, side 1 in the high half) padded to 16 bytes; u32 keys [4 x key
// buckets].
#include "logf_replay.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace rb200;

namespace
{

float arg_of(uint32_t v)
{
    const float p = std::fmaf(static_cast<float>(v), 2.3283064e-10f, 2.3283064e-10f);
    const float x = 2.0f * p - 1.0f;
    return (1.0f - x) * (1.0f + x);
}

// Cuckoo insertion into 2^lb buckets of four; false when a key finds no place.
bool build_keys(const std::vector<uint32_t>& members, uint32_t lb, std::vector<uint32_t>& keys)
{
    keys.assign(4ull << lb, 0u);
    uint64_t rng = 0x243F6A8885A308D3ull;
    for(uint32_t key : members)
    {
        uint32_t cur = key;
        bool     placed = false;
        for(int kick = 0; kick < 2000 && !placed; kick++)
        {
            const uint32_t h[2] = {lr::bucket1(cur, lb), lr::bucket2(cur, lb)};
            for(int c = 0; c < 2 && !placed; c++)
                for(int s = 0; s < 4 && !placed; s++)
                    if(keys[4 * h[c] + s] == 0u)
                    {
                        keys[4 * h[c] + s] = cur;
                        placed             = true;
                    }
            if(placed)
                break;
            // evict a random key of one of the two buckets; it moves to its other bucket
            rng ^= rng << 13;
            rng ^= rng >> 7;
            rng ^= rng << 17;
            const uint32_t slot = 4 * h[rng & 1] + static_cast<uint32_t>((rng >> 1) & 3);
            std::swap(cur, keys[slot]);
        }
        if(!placed)
            return false;
    }
    return true;
}

} // namespace

int main(int argc, char** argv)
{
    if(argc != 2)
    {
        std::fprintf(stderr, "usage: %s out.bin\n", argv[0]);
        return 2;
    }
    // 1. reachable arguments, as a bitmap over float bit patterns
    std::vector<uint64_t> seen((1ull << 32) / 64, 0);
#pragma omp parallel for schedule(static)
    for(long long hi = 0; hi < 65536; hi++)
    {
        for(uint32_t lo = 0; lo < 65536; lo++)
        {
            const uint32_t b = lr::fbits(arg_of(static_cast<uint32_t>(hi << 16 | lo)));
            __atomic_fetch_or(&seen[b >> 6], 1ull << (b & 63), __ATOMIC_RELAXED);
        }
    }
    std::vector<uint32_t> args;
    for(size_t w = 0; w < seen.size(); w++)
        for(uint64_t m = seen[w]; m; m &= m - 1)
            args.push_back(static_cast<uint32_t>(w * 64 + __builtin_ctzll(m)));
    seen.clear();
    seen.shrink_to_fit();

    // 2. differences between the host's logf and the kernels' rounding
    const size_t          na = args.size();
    std::vector<uint32_t> host(na), dist(na, 0), side(na, 0);
    std::vector<uint8_t>  state(na, 0); // 0 same, 1 member, 2 not in range, 3 not the neighbour
#pragma omp parallel for schedule(dynamic, 4096)
    for(long long i = 0; i < static_cast<long long>(na); i++)
    {
        const float t = lr::ffrom(args[i]);
        host[i]       = lr::fbits(::logf(t));
        if(!(t >= 0x1p-64f) || !(t <= 1.0f))
        {
            state[i] = lr::fbits(pm::logf(t)) != host[i] ? 2 : 0;
            continue;
        }
        uint32_t    d, s;
        const float f = lr::base(t, d, s);
        dist[i]       = d;
        side[i]       = s;
        if(lr::fbits(f) == host[i])
            continue;
        const uint32_t fb = lr::fbits(f);
        const uint32_t nb = (s != 0u) == ((fb >> 31) == 0u) ? fb + 1u : fb - 1u;
        state[i]          = nb == host[i] ? 1 : 3;
    }
    std::vector<uint32_t> bound(lr::kBuckets, 0);
    std::vector<uint32_t> members;
    for(size_t i = 0; i < na; i++)
    {
        if(state[i] >= 2)
        {
            std::fprintf(stderr, "argument %08x: %s\n", args[i],
                         state[i] == 2 ? "outside [2^-64, 1] differs from the host"
                                       : "the host's result is not the neighbour on the logarithm's side");
            return 1;
        }
        if(state[i] == 0)
            continue;
        const uint32_t key = args[i] >> lr::kBucketShift;
        const uint32_t b   = dist[i] + 1u;
        if(key >= lr::kBuckets || b > 65535u)
        {
            std::fprintf(stderr, "argument %08x: bucket %u, bound %u out of range\n", args[i], key, b);
            return 1;
        }
        const uint32_t sh  = side[i] ? 16 : 0;
        const uint32_t cur = (bound[key] >> sh) & 0xffffu;
        if(b > cur)
            bound[key] = (bound[key] & ~(0xffffu << sh)) | (b << sh);
        members.push_back(args[i]);
    }

    // 3. the member set: key buckets at a load of at most 1/2
    uint32_t lb = 1;
    while((4ull << lb) < 2 * members.size())
        lb++;
    std::vector<uint32_t> keys;
    while(!build_keys(members, lb, keys))
        lb++;

    // 4. replay every reachable argument through the kernels' code
    lr::Table tb;
    tb.bound        = bound.data();
    tb.keys         = reinterpret_cast<const uint4*>(keys.data());
    tb.log2_buckets = lb;
    long long bad = 0, probed = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : bad, probed)
    for(long long i = 0; i < static_cast<long long>(na); i++)
    {
        const float t = lr::ffrom(args[i]);
        if(lr::fbits(lr::logf_host(t, tb)) != host[i])
            bad++;
        if(t >= 0x1p-64f && t <= 1.0f)
        {
            const uint32_t b = (bound[args[i] >> lr::kBucketShift] >> (side[i] ? 16 : 0)) & 0xffffu;
            probed += dist[i] < b ? 1 : 0;
        }
    }
    std::printf("logf replay: %zu reachable arguments, %zu differ from the kernels' rounding "
                "(%.3f%%), %.2f%% looked up, %u key buckets, %lld mismatches\n",
                na, members.size(), 100.0 * members.size() / na, 100.0 * probed / na, 1u << lb, bad);
    if(bad != 0)
        return 1;

    FILE* f = std::fopen(argv[1], "wb");
    if(!f)
        return 1;
    const uint32_t hdr[6] = {static_cast<uint32_t>(lr::kBucketShift), lr::kBuckets, lb,
                             static_cast<uint32_t>(members.size()), static_cast<uint32_t>(na), 0u};
    std::fwrite("RBLOGF02", 1, 8, f);
    std::fwrite(hdr, 4, 6, f);
    std::fwrite(bound.data(), 4, bound.size(), f);
    const size_t pad      = (16 - (8 + 24 + 4 * bound.size()) % 16) % 16;
    const char   zero[16] = {};
    std::fwrite(zero, 1, pad, f);
    std::fwrite(keys.data(), 4, keys.size(), f);
    return std::fclose(f) == 0 ? 0 : 1;
}
