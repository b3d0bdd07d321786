// threefry.cu -- ThreeFry 2x32-20, 2x64-20, 4x32-20 and 4x64-20 generators.
//
// Same output contract as philox.cu, generalised to a block of D words of W bits
// (library/src/rng/threefry.hpp:86-198): vector j holds the distribution applied to the
// D stream words starting at
//     p(j) = D*j + (j % 262144 == 0 ? start0 : floor(head/ow)*iw),
// where start0 = ceil(head/ow)*iw is what the head consumed on thread 0 of the reference's
// 1024x256 grid (threefry.hpp:121-123); head and tail run sequentially, and the engine
// advances by ceil(n/ow)*iw words per call (threefry.hpp:381-386).
//
// The block function is the Threefish-style round schedule of
// library/include/rocrand/rocrand_threefry{2,4}_impl.h: 20 rounds of add/rotate/xor with
// the Skein rotation constants and a key injection every 4 rounds.  The injected key words
// (including the +round counter) are folded on the host into 6 per-launch key vectors.
#include "common.hpp"
#include "dist.cuh"
#include "generators.hpp"
#include "host_exec.hpp"
#include "launch.cuh"
#include "poisson.hpp"

#include <cstring>
#include <type_traits>

namespace rb200
{

template<class W>
__host__ __device__ __forceinline__ W rotl(W x, int d)
{
    constexpr int B = 8 * sizeof(W);
    return (x << (d & (B - 1))) | (x >> ((B - d) & (B - 1)));
}

// Rotation of round r, lane k: the Skein/Random123 constants of
// rocrand_threefry4_impl.h:62-92 and rocrand_threefry2_impl.h:70-93 (compile-time after
// unrolling).
template<class W, int D>
__host__ __device__ constexpr int rot_of(int r, int k)
{
    constexpr int r32x4[8][2] = {{10, 26}, {11, 21}, {13, 27}, {23, 5},
                                 {6, 20},  {17, 11}, {25, 10}, {18, 20}};
    constexpr int r64x4[8][2] = {{14, 16}, {52, 57}, {23, 40}, {5, 37},
                                 {25, 33}, {46, 12}, {58, 22}, {32, 32}};
    constexpr int r32x2[8]    = {13, 15, 26, 6, 17, 29, 16, 24};
    constexpr int r64x2[8]    = {16, 42, 12, 31, 16, 32, 24, 21};
    if(D == 4)
        return sizeof(W) == 4 ? r32x4[r & 7][k] : r64x4[r & 7][k];
    return sizeof(W) == 4 ? r32x2[r & 7] : r64x2[r & 7];
}

template<class W, int D>
struct TfBlock
{
    W w[D];
};

// Key vectors: kv[0] is added before round 0, kv[1 + i] after round 4*i + 3.
template<class W, int D>
struct TfKeys
{
    W kv[6][D];
};

template<class W, int D>
TfKeys<W, D> threefry_keys(const W (&key)[D])
{
    W ks[D + 1];
    ks[D] = sizeof(W) == 4 ? static_cast<W>(0x1BD11BDAu) : static_cast<W>(0x1BD11BDAA9FC1A22ull);
    for(int i = 0; i < D; i++)
    {
        ks[i] = key[i];
        ks[D] ^= key[i];
    }
    TfKeys<W, D> t;
    for(int i = 0; i < D; i++)
        t.kv[0][i] = ks[i];
    for(int inj = 0; inj < 5; inj++)
        for(int i = 0; i < D; i++)
            t.kv[1 + inj][i] = ks[(i + 1 + inj) % (D + 1)] + (i == D - 1 ? static_cast<W>(1 + inj) : 0);
    return t;
}

template<class W, int D>
__host__ __device__ __forceinline__ TfBlock<W, D> threefry_block(TfBlock<W, D> x, const TfKeys<W, D>& k)
{
#pragma unroll
    for(int i = 0; i < D; i++)
        x.w[i] += k.kv[0][i];
#pragma unroll
    for(int r = 0; r < 20; r++)
    {
        if constexpr(D == 4)
        {
            if((r & 2) == 0)
            {
                x.w[0] += x.w[1];
                x.w[1] = rotl(x.w[1], rot_of<W, D>(r, 0));
                x.w[1] ^= x.w[0];
                x.w[2] += x.w[3];
                x.w[3] = rotl(x.w[3], rot_of<W, D>(r, 1));
                x.w[3] ^= x.w[2];
            }
            else
            {
                x.w[0] += x.w[3];
                x.w[3] = rotl(x.w[3], rot_of<W, D>(r, 0));
                x.w[3] ^= x.w[0];
                x.w[2] += x.w[1];
                x.w[1] = rotl(x.w[1], rot_of<W, D>(r, 1));
                x.w[1] ^= x.w[2];
            }
        }
        else
        {
            x.w[0] += x.w[1];
            x.w[1] = rotl(x.w[1], rot_of<W, D>(r, 0));
            x.w[1] ^= x.w[0];
        }
        if((r & 3) == 3)
        {
#pragma unroll
            for(int i = 0; i < D; i++)
                x.w[i] += k.kv[1 + r / 4][i];
        }
    }
    return x;
}

// Counter + 64-bit addend, carries through every word (discard_state of each engine; for
// 64-bit words the addend is the low word only).
template<class W, int D>
__host__ __device__ __forceinline__ TfBlock<W, D> tf_add(TfBlock<W, D> c, unsigned long long a)
{
    if constexpr(sizeof(W) == 8)
    {
        const W old = c.w[0];
        c.w[0] += a;
        W carry = c.w[0] < old ? 1 : 0;
#pragma unroll
        for(int i = 1; i < D; i++)
        {
            const W o = c.w[i];
            c.w[i] += carry;
            carry = (carry && c.w[i] < o) ? 1 : 0;
        }
    }
    else
    {
        // low two words as one 64-bit value, then the carry into the rest
        const unsigned long long lo  = (static_cast<unsigned long long>(c.w[1]) << 32) | c.w[0];
        const unsigned long long nlo = lo + a;
        c.w[0]                       = static_cast<W>(nlo);
        c.w[1]                       = static_cast<W>(nlo >> 32);
        if constexpr(D == 4)
        {
            if(nlo < lo)
            {
                c.w[2] += 1;
                if(c.w[2] == 0)
                    c.w[3] += 1;
            }
        }
    }
    return c;
}

// Engine position: word index = D * counter + sub.
template<class W, int D>
struct TfPos
{
    TfBlock<W, D> counter{};
    uint32_t      sub = 0;
    void          advance(unsigned long long k)
    {
        const unsigned long long q = sub + (k % D);
        counter                    = tf_add(counter, k / D + q / D);
        sub                        = static_cast<uint32_t>(q % D);
    }
};

// Words s..s+D-1 of the concatenation (a, b): the engine's interleave.
template<class W, int D>
__host__ __device__ __forceinline__ TfBlock<W, D> tf_interleave(const TfBlock<W, D>& a, const TfBlock<W, D>& b,
                                                       uint32_t s)
{
    TfBlock<W, D> m;
    if constexpr(D == 2)
    {
        m.w[0] = a.w[1];
        m.w[1] = b.w[0];
    }
    else
    {
        switch(s)
        {
            case 1: m = TfBlock<W, D>{{a.w[1], a.w[2], a.w[3], b.w[0]}}; break;
            case 2: m = TfBlock<W, D>{{a.w[2], a.w[3], b.w[0], b.w[1]}}; break;
            default: m = TfBlock<W, D>{{a.w[3], b.w[0], b.w[1], b.w[2]}}; break;
        }
    }
    return m;
}

template<class W, int D>
struct TfCall
{
    TfKeys<W, D>       keys;
    TfBlock<W, D>      c0;
    uint32_t           s0;
    uint32_t           adj;    // floor(head/ow)*iw: stream offset of vectors j % 262144 != 0
    uint32_t           start0; // ceil(head/ow)*iw: stream offset of vectors j % 262144 == 0
    uint32_t           head, tail;
    unsigned char*     data;
    unsigned char*     vec;
    unsigned long long n, vec_n;
};

template<class W, int D>
__host__ __device__ __forceinline__ W tf_word(const TfCall<W, D>& a, unsigned long long p)
{
    const unsigned long long q = a.s0 + p;
    const TfBlock<W, D>      b = threefry_block(tf_add(a.c0, q / D), a.keys);
    W                        r = b.w[0];
#pragma unroll
    for(int i = 1; i < D; i++)
        if(static_cast<int>(q % D) == i)
            r = b.w[i];
    return r;
}

template<class W, int D, class F>
__host__ __device__ void tf_scalar_run(const TfCall<W, D>& a, const F& f, unsigned long long pos,
                              typename F::T* out, uint32_t count)
{
    typename F::T v[F::ow];
    W             in[F::iw];
    for(uint32_t done = 0; done < count; done += F::ow)
    {
        for(unsigned i = 0; i < F::iw; i++)
            in[i] = tf_word(a, pos++);
        f(in, v);
        for(unsigned o = 0; o < F::ow && done + o < count; o++)
            out[done + o] = v[o];
    }
}

// Stores one output vector of VB bytes (8, 16 or 32) from an array of T.
template<class T, unsigned N>
__device__ __forceinline__ void store_vec(unsigned char* p, const T (&v)[N])
{
    constexpr unsigned VB = sizeof(T) * N;
    uint32_t           w[VB / 4];
    memcpy(w, v, VB);
    if constexpr(VB == 8)
        __stcs(reinterpret_cast<uint2*>(p), make_uint2(w[0], w[1]));
    else if constexpr(VB == 16)
        __stcs(reinterpret_cast<uint4*>(p), make_uint4(w[0], w[1], w[2], w[3]));
    else
    {
        static_assert(VB == 32, "vector size");
        __stcs(reinterpret_cast<uint4*>(p), make_uint4(w[0], w[1], w[2], w[3]));
        __stcs(reinterpret_cast<uint4*>(p) + 1, make_uint4(w[4], w[5], w[6], w[7]));
    }
}

template<class W, int D, class F, bool kAligned>
__global__ void __launch_bounds__(kBlock) threefry_fill(TfCall<W, D> a, F f)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const F g = stage_table(f, smem);

    constexpr unsigned opt = D / F::iw;
    constexpr unsigned VB  = opt * F::ow * sizeof(typename F::T);
    const unsigned long long tid    = static_cast<unsigned long long>(blockIdx.x) * kBlock + threadIdx.x;
    const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * kBlock;

    for(unsigned long long j = tid; j < a.vec_n; j += stride)
    {
        TfBlock<W, D> b;
        if(kAligned)
        {
            b = threefry_block(tf_add(a.c0, (a.s0 + a.adj) / D + j), a.keys);
        }
        else
        {
            const unsigned long long q = a.s0 + ((j & (kPhiloxRefStride - 1)) == 0 ? a.start0 : a.adj) + D * j;
            const TfBlock<W, D>      c = tf_add(a.c0, q / D);
            const uint32_t           s = static_cast<uint32_t>(q % D);
            b                          = threefry_block(c, a.keys);
            if(s != 0)
                b = tf_interleave(b, threefry_block(tf_add(c, 1), a.keys), s);
        }
        typename F::T out[opt * F::ow];
#pragma unroll
        for(unsigned s = 0; s < opt; s++)
            g(b.w + s * F::iw, out + s * F::ow);
        store_vec(a.vec + j * VB, out);
    }

    if(tid == 0)
    {
        using T = typename F::T;
        if(a.head > 0)
            tf_scalar_run(a, g, 0, reinterpret_cast<T*>(a.data), a.head);
        if(a.tail > 0)
        {
            const unsigned long long pos
                = D * a.vec_n + ((a.vec_n % kPhiloxRefStride) == 0 ? a.start0 : a.adj);
            tf_scalar_run(a, g, pos, reinterpret_cast<T*>(a.data) + (a.n - a.tail), a.tail);
        }
    }
}

// The same output contract on the host (host generators without a GPU): every vector by the
// general rule of threefry_fill, the head and tail by the same sequential run.
template<class W, int D, class F>
static void threefry_run_host(const TfCall<W, D>& a, const F& f)
{
    constexpr unsigned opt = D / F::iw;
    constexpr unsigned VB  = opt * F::ow * sizeof(typename F::T);
    host_parallel_for(a.vec_n, [&](unsigned long long j0, unsigned long long j1) {
        for(unsigned long long j = j0; j < j1; j++)
        {
            const unsigned long long q = a.s0 + ((j & (kPhiloxRefStride - 1)) == 0 ? a.start0 : a.adj) + D * j;
            const TfBlock<W, D>      c = tf_add(a.c0, q / D);
            const uint32_t           s = static_cast<uint32_t>(q % D);
            TfBlock<W, D>            b = threefry_block(c, a.keys);
            if(s != 0)
                b = tf_interleave(b, threefry_block(tf_add(c, 1), a.keys), s);
            typename F::T out[opt * F::ow];
            for(unsigned k = 0; k < opt; k++)
                f(b.w + k * F::iw, out + k * F::ow);
            std::memcpy(a.vec + j * VB, out, VB);
        }
    });
    using T = typename F::T;
    if(a.head > 0)
        tf_scalar_run(a, f, 0, reinterpret_cast<T*>(a.data), a.head);
    if(a.tail > 0)
    {
        const unsigned long long pos = D * a.vec_n + ((a.vec_n % kPhiloxRefStride) == 0 ? a.start0 : a.adj);
        tf_scalar_run(a, f, pos, reinterpret_cast<T*>(a.data) + (a.n - a.tail), a.tail);
    }
}

// ---------------------------------------------------------------------------------------

template<class W, int D, rocrand_rng_type kType>
class ThreefryGenerator final : public PseudoGeneratorBase
{
public:
    rocrand_rng_type type() const override { return kType; }
    bool             set_host_execution() override { return enable_host(); }

    // Output `index` of distribution d comes from engine word index * iw / ow (index a
    // multiple of ow, output aligned to the distribution's vector): that offset.
    rocrand_status set_output_position(Dist d, unsigned long long index) override
    {
        if(sizeof(W) == 4 && d == Dist::U64)
            return ROCRAND_STATUS_TYPE_ERROR;
        DistParams p;
        auto body = [&](auto f) -> rocrand_status {
            using F = decltype(f);
            if constexpr(D % F::iw != 0)
                return ROCRAND_STATUS_TYPE_ERROR;
            else
            {
                if(index % F::ow != 0)
                    return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
                return set_offset(index / F::ow * F::iw);
            }
        };
        if constexpr(sizeof(W) == 8)
            return with_functor64(d, p, body);
        else
        {
            if constexpr(D == 2)
            {
                if(d == Dist::NORMAL_F64 || d == Dist::LOGNORMAL_F64)
                    return body(FnNormalD1{p.mean_d, p.std_d, false});
            }
            return with_functor(d, p, body);
        }
    }

    rocrand_status init() override
    {
        if(m_initialized)
            return ROCRAND_STATUS_SUCCESS;
        // the Poisson tables are allocated here, as the reference's generators do in init(), so
        // that a generate call recorded by a stream capture allocates nothing
        if(m_poisson.reserve() != ROCRAND_STATUS_SUCCESS)
            return ROCRAND_STATUS_ALLOCATION_FAILED;
        // seed(seed, 0, offset): key from the seed (rocrand_threefry{2,4}x{32,64}_20.h seed())
        if constexpr(D == 4)
        {
            for(int i = 0; i < 4; i++)
                m_key[i] = static_cast<W>(m_seed >> (16 * i));
        }
        else
        {
            m_key[0] = static_cast<W>(m_seed);
            m_key[1] = static_cast<W>(m_seed >> 32);
        }
        m_keys = threefry_keys<W, D>(m_key);
        m_pos  = TfPos<W, D>{};
        m_pos.advance(m_offset);
        m_initialized = true;
        return ROCRAND_STATUS_SUCCESS;
    }

    rocrand_status set_order(rocrand_ordering order) override
    {
        switch(order)
        {
            case ROCRAND_ORDERING_PSEUDO_DEFAULT:
            case ROCRAND_ORDERING_PSEUDO_DYNAMIC:
            case ROCRAND_ORDERING_PSEUDO_BEST:
            case ROCRAND_ORDERING_PSEUDO_LEGACY:
                m_order       = order;
                m_initialized = false;
                return ROCRAND_STATUS_SUCCESS;
            default: return ROCRAND_STATUS_OUT_OF_RANGE;
        }
    }

    rocrand_status generate(void* data, size_t n, Dist d, const DistParams& p) override
    {
        if constexpr(sizeof(W) == 4)
        {
            if(d == Dist::U64)
                return ROCRAND_STATUS_TYPE_ERROR; // threefry.hpp:316-321
        }
        rocrand_status st = init();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        if(data == nullptr)
            return ROCRAND_STATUS_SUCCESS;
        const size_t tsize = dist_elem_size(d);
        if(reinterpret_cast<uintptr_t>(data) % tsize != 0)
            return ROCRAND_STATUS_LENGTH_NOT_MULTIPLE;
        auto body = [&](auto f) -> rocrand_status {
            using F = decltype(f);
            if constexpr(D % F::iw != 0)
                return ROCRAND_STATUS_TYPE_ERROR;
            else
                return run(f, data, n, tsize);
        };
        if constexpr(sizeof(W) == 8)
            return with_functor64(d, p, body);
        else
        {
            // ThreeFry2x32 serves double normals with the one-word inverse-erf functor
            // (threefry.hpp:441-449).
            if constexpr(D == 2)
            {
                if(d == Dist::NORMAL_F64)
                    return body(FnNormalD1{p.mean_d, p.std_d, false});
                if(d == Dist::LOGNORMAL_F64)
                    return body(FnNormalD1{p.mean_d, p.std_d, true});
            }
            return with_functor(d, p, body);
        }
    }

    rocrand_status generate_poisson(unsigned int* data, size_t n, double lambda) override
    {
        rocrand_status st = init();
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        DistParams p;
        st = m_poisson.get(lambda, m_stream, false, p);
        if(st != ROCRAND_STATUS_SUCCESS)
            return st;
        return generate(data, n, Dist::POISSON, p);
    }

private:
    template<class F>
    rocrand_status run(const F& f, void* data, size_t n, size_t tsize)
    {
        constexpr unsigned iw  = F::iw;
        constexpr unsigned ow  = F::ow;
        constexpr unsigned fow = (D / iw) * ow;
        const uintptr_t    addr = reinterpret_cast<uintptr_t>(data);
        const size_t       mis  = (fow - addr / tsize % fow) % fow;
        TfCall<W, D>       a;
        a.keys   = m_keys;
        a.c0     = m_pos.counter;
        a.s0     = m_pos.sub;
        a.head   = static_cast<uint32_t>(n < mis ? n : mis);
        a.tail   = static_cast<uint32_t>((n - a.head) % fow);
        a.vec_n  = (n - a.head) / fow;
        a.adj    = a.head / ow * iw;
        a.start0 = (a.head + ow - 1) / ow * iw;
        a.n      = n;
        a.data   = static_cast<unsigned char*>(data);
        a.vec    = a.data + mis * tsize;
        if(n == 0)
            return ROCRAND_STATUS_SUCCESS;
        if(m_host_exec)
        {
            threefry_run_host(a, f);
            m_pos.advance(static_cast<unsigned long long>((n + ow - 1) / ow) * iw);
            return ROCRAND_STATUS_SUCCESS;
        }
        const size_t             smem    = table_smem_bytes(f);
        const bool               aligned = a.start0 == a.adj && ((a.s0 + a.adj) % D) == 0;
        const unsigned long long work    = a.vec_n > 0 ? a.vec_n : 1;
        if(aligned)
        {
            auto k = threefry_fill<W, D, F, true>;
            k<<<grid_for(k, work, smem), kBlock, smem, m_stream>>>(a, f);
        }
        else
        {
            auto k = threefry_fill<W, D, F, false>;
            k<<<grid_for(k, work, smem), kBlock, smem, m_stream>>>(a, f);
        }
        const rocrand_status s = launch_status();
        if(s == ROCRAND_STATUS_SUCCESS)
            m_pos.advance(static_cast<unsigned long long>((n + ow - 1) / ow) * iw);
        return s;
    }

    W            m_key[D] = {};
    TfKeys<W, D> m_keys{};
    TfPos<W, D>  m_pos;
};

rocrand_generator_base_type* make_threefry(rocrand_rng_type t)
{
    switch(t)
    {
        case ROCRAND_RNG_PSEUDO_THREEFRY2_32_20:
            return new ThreefryGenerator<uint32_t, 2, ROCRAND_RNG_PSEUDO_THREEFRY2_32_20>();
        case ROCRAND_RNG_PSEUDO_THREEFRY2_64_20:
            return new ThreefryGenerator<unsigned long long, 2, ROCRAND_RNG_PSEUDO_THREEFRY2_64_20>();
        case ROCRAND_RNG_PSEUDO_THREEFRY4_32_20:
            return new ThreefryGenerator<uint32_t, 4, ROCRAND_RNG_PSEUDO_THREEFRY4_32_20>();
        case ROCRAND_RNG_PSEUDO_THREEFRY4_64_20:
            return new ThreefryGenerator<unsigned long long, 4, ROCRAND_RNG_PSEUDO_THREEFRY4_64_20>();
        default: return nullptr;
    }
}

} // namespace rb200
