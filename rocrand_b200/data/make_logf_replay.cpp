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
// 2. For each distinct t, the host's logf(t) against the kernels' own rounding f of the
//    accurate logarithm (logf_replay.cuh base(), compiled here for the host: the same IEEE
//    operations).  Where they differ, the argument and the host's result are stored, and
//    the argument's bucket bound is raised to its distance from the rounding boundary.
// 3. Every t is replayed through logf_replay.cuh logf_host() with the finished table and
//    must give the host's logf(t) bit for bit; otherwise nothing is written.
//
// Output (little-endian): "RBLOGF01", u32 bucket shift, u32 bucket count, u32 log2 of the
// slot count, u32 longest probe, u32 stored arguments, u32 reachable arguments, u16 bounds
// [bucket count] padded to 16 bytes, u32 slot pairs (argument bits, result bits)[slots].
#include "logf_replay.cuh"

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
    std::vector<uint32_t> host(na);
    std::vector<uint8_t>  differs(na, 0);
    std::vector<uint32_t> dist(na, 0);
#pragma omp parallel for schedule(dynamic, 4096)
    for(long long i = 0; i < static_cast<long long>(na); i++)
    {
        const float t = lr::ffrom(args[i]);
        host[i]       = lr::fbits(::logf(t));
        if(!(t > 0.0f) || !(t <= 1.0f))
        {
            differs[i] = lr::fbits(pm::logf(t)) != host[i] ? 2 : 0; // must not happen
            continue;
        }
        uint32_t    d;
        const float f = lr::base(t, d);
        dist[i]       = d;
        differs[i]    = lr::fbits(f) != host[i] ? 1 : 0;
    }
    std::vector<uint16_t> bound(lr::kBuckets, 0);
    std::vector<size_t>   stored;
    for(size_t i = 0; i < na; i++)
    {
        if(differs[i] == 2)
        {
            std::fprintf(stderr, "argument %08x outside (0, 1] differs from the host\n", args[i]);
            return 1;
        }
        if(differs[i] == 0)
            continue;
        const uint32_t key = args[i] >> lr::kBucketShift;
        const double   b   = static_cast<double>(dist[i]) + 1.0;
        if(key >= lr::kBuckets || b > 65535.0)
        {
            std::fprintf(stderr, "argument %08x: bucket %u, bound %.1f out of range\n", args[i], key, b);
            return 1;
        }
        bound[key] = std::max<uint16_t>(bound[key], static_cast<uint16_t>(b));
        stored.push_back(i);
    }

    // open-addressing hash table at load <= 1/2
    uint32_t log2s = 1;
    while((1ull << log2s) < 2 * stored.size())
        log2s++;
    const uint32_t        mask = (1u << log2s) - 1u;
    std::vector<uint32_t> slots(2ull << log2s, 0);
    uint32_t              max_probe = 0;
    for(size_t i : stored)
    {
        const uint32_t key = args[i];
        uint32_t       h   = (key * lr::kHashMul) >> (32 - log2s);
        uint32_t       k   = 1;
        while(slots[2 * h] != 0)
        {
            h = (h + 1u) & mask;
            k++;
        }
        slots[2 * h]     = key;
        slots[2 * h + 1] = host[i];
        max_probe        = std::max(max_probe, k);
    }

    // 3. replay every reachable argument through the kernels' code
    lr::Table tb;
    tb.bound      = bound.data();
    tb.slots      = slots.data();
    tb.log2_slots = log2s;
    tb.max_probe  = max_probe;
    long long bad = 0, probed = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : bad, probed)
    for(long long i = 0; i < static_cast<long long>(na); i++)
    {
        const float t = lr::ffrom(args[i]);
        if(lr::fbits(lr::logf_host(t, tb)) != host[i])
            bad++;
        if(t > 0.0f && t <= 1.0f)
        {
            const uint16_t b = bound[args[i] >> lr::kBucketShift];
            probed += (b != 0 && dist[i] <= b) ? 1 : 0;
        }
    }
    std::printf("logf replay: %zu reachable arguments, %zu differ from the kernels' rounding "
                "(%.3f%%), %.2f%% looked up, %u slots, longest probe %u, %lld mismatches\n",
                na, stored.size(), 100.0 * stored.size() / na, 100.0 * probed / na, mask + 1u,
                max_probe, bad);
    if(bad != 0)
        return 1;

    FILE* f = std::fopen(argv[1], "wb");
    if(!f)
        return 1;
    const uint32_t hdr[6] = {static_cast<uint32_t>(lr::kBucketShift), lr::kBuckets, log2s, max_probe,
                             static_cast<uint32_t>(stored.size()), static_cast<uint32_t>(na)};
    std::fwrite("RBLOGF01", 1, 8, f);
    std::fwrite(hdr, 4, 6, f);
    std::fwrite(bound.data(), 2, bound.size(), f);
    const size_t pad = (16 - (8 + 24 + 2 * bound.size()) % 16) % 16;
    const char   zero[16] = {};
    std::fwrite(zero, 1, pad, f);
    std::fwrite(slots.data(), 4, slots.size(), f);
    return std::fclose(f) == 0 ? 0 : 1;
}
