// CPU gang port of Loom's compact and hybrid SIMD backends, with a
// multi-worker harness in the manner of Loom's mp::Shop.
//
// BASELINE INFRASTRUCTURE ONLY.  bench.py's CPU leg and tests/ run it
// (oracle/build_gang.py builds oracle/_lib/libloomgang.so); the product never
// does.  Loom's own compact/hybrid backends (src/vm/simd.hpp) need clang's
// elementwise builtins and range-v3 (src/vm/bve.hpp:30-34), which this
// machine does not have, so this header restates their algorithm in plain
// C++20 for g++; the per-kernel block code comes from oracle/gang_emit.py.
//
// What is restated, with the Loom code it follows:
//  * threaded block dispatch (threaded_dispatch::eval, simd.hpp:3577-3727):
//    run a block for the lanes standing at it, drop it from the pending set,
//    add every successor that has lanes, and go on into the successor with
//    the most lanes (the first in jump-table order on a tie) while that
//    group is larger than the threshold;
//  * major_group (simd.hpp:2640-2670): among candidate blocks in ascending
//    order, the one with strictly the most lanes; greedy_groups (2480-2530):
//    the blocks some non-halted lane stands at;
//  * compact execution (compact_compiler, use_tbd, simd.hpp:3850-3880): a
//    gang from block 0 with threshold 0, then the largest pending group
//    until every lane has halted;
//  * hybrid execution (hybrid_compiler::visitor, simd.hpp:4105-4180): the
//    stream's threads in aligned chunks of N up to the first halted one;
//    per chunk the largest group, dispatch while its group exceeds
//    t = ceil(N * UTR) (0 once the visited view is no larger than
//    align_up(ceil(C * blocks * UTR), C) or C), the pending set, else the
//    largest group again; then a stable counting sort by PC with the halted
//    threads last (counting_sort, simd.hpp:2680-2745), and the halted rows
//    from align_up(size - halted, C) on exchanged for new inputs once at
//    least C threads have halted (ConcurrentStreamFacade, simd.hpp:2803-2905);
//  * mp::Shop (src/vm/mp.hpp:316-385): one stream per worker thread, each
//    exchanging finished threads for new inputs; here the workers draw
//    inputs from one shared cursor.
#pragma once

#include <atomic>
#include <bit>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <immintrin.h>
#include <thread>
#include <vector>

namespace loom_gang
{
// ---- instruction semantics (Loom src/vm/operators.hpp, as the scalar
// backend bse evaluates them on the host)

template <typename To, typename From>
inline To
bitcast(const From v)
{
    static_assert(sizeof(To) == sizeof(From), "bitcast needs equal sizes");
    To r;
    std::memcpy(&r, &v, sizeof(To));
    return r;
}

// std::max / std::min
template <typename T>
inline T
op_max(const T a, const T b)
{
    return (a < b) ? b : a;
}
template <typename T>
inline T
op_min(const T a, const T b)
{
    return (b < a) ? b : a;
}

inline float op_abs(float v) { return std::fabs(v); }
inline double op_abs(double v) { return std::fabs(v); }
inline int op_abs(int v) { return v < 0 ? -v : v; }
inline long long op_abs(long long v) { return v < 0 ? -v : v; }
inline float op_round(float v) { return std::round(v); }
inline double op_round(double v) { return std::round(v); }
inline float op_ceil(float v) { return std::ceil(v); }
inline double op_ceil(double v) { return std::ceil(v); }
inline float op_floor(float v) { return std::floor(v); }
inline double op_floor(double v) { return std::floor(v); }
inline float op_trunc(float v) { return std::trunc(v); }
inline double op_trunc(double v) { return std::trunc(v); }
inline float op_sqrt(float v) { return std::sqrt(v); }
inline double op_sqrt(double v) { return std::sqrt(v); }
// the host libm, per lane, as bse calls it
inline float op_sin(float v) { return std::sin(v); }
inline double op_sin(double v) { return std::sin(v); }
inline float op_cos(float v) { return std::cos(v); }
inline double op_cos(double v) { return std::cos(v); }
inline float op_copysign(float a, float b) { return std::copysign(a, b); }
inline double op_copysign(double a, double b) { return std::copysign(a, b); }
inline float op_fma(float x, float y, float z) { return std::fma(x, y, z); }
inline double op_fma(double x, double y, double z) { return std::fma(x, y, z); }
inline float op_rsqrt(float v) { return 1.0f / std::sqrt(v); }
inline double op_rsqrt(double v) { return 1.0 / std::sqrt(v); }

// spellings of non-finite literals in the shared lowering
inline float __uint_as_float(const unsigned u) { return bitcast<float>(u); }
inline double __longlong_as_double(const long long u) { return bitcast<double>(u); }

/// The launch's table (the tab op, a Loom extension of this project).
struct Cols
{
    const unsigned* table;
};

struct Ctx
{
    const Cols* cols;
};

template <typename T>
inline T
table_load(const Cols& c, const unsigned idx)
{
    return bitcast<T>(c.table[idx]);
}

/// assert_fp aborts bse on NaN or infinity; the port passes the value on.
template <typename T>
inline T
op_assert_fp(const T v, const Ctx&)
{
    return v;
}

enum Method
{
    kCompact = 0,
    kHybrid  = 1,
};

// ---- gang execution

/// Gang block executions and the lanes active in them.
struct Counters
{
    std::uint64_t blocks = 0;
    std::uint64_t lanes  = 0;
};

/// Bit l set when lane l of an N-lane gang stands at block b (an AVX-512
/// compare per 16 lanes; the PCs are 32-bit).
template <int N>
inline std::uint64_t
lanes_at(const int* pc, const int b)
{
    if constexpr(N == 8)
        return _mm256_cmpeq_epi32_mask(_mm256_load_si256(reinterpret_cast<const __m256i*>(pc)), _mm256_set1_epi32(b));
    else if constexpr(N % 16 == 0)
    {
        std::uint64_t m = 0;
        for(int i = 0; i < N / 16; ++i)
            m |= static_cast<std::uint64_t>(_mm512_cmpeq_epi32_mask(_mm512_load_si512(pc + 16 * i), _mm512_set1_epi32(b)))
                 << (16 * i);
        return m;
    }
    else
    {
        std::uint64_t m = 0;
        for(int l = 0; l < N; ++l) m |= static_cast<std::uint64_t>(pc[l] == b) << l;
        return m;
    }
}

/// Lanes of an N-lane gang at block b.
template <int N>
inline unsigned
pops_at(const int* pc, const int b)
{
    return static_cast<unsigned>(std::popcount(lanes_at<N>(pc, b)));
}

template <typename G>
struct Gang
{
    static constexpr int N    = G::N;
    static constexpr int NB   = G::kNumBlocks;
    static constexpr int HALT = NB;
    using Regs                = typename G::Regs;
    using Counters            = loom_gang::Counters;

    static std::uint64_t
    lanes_at(const Regs& R, const int b)
    {
        return loom_gang::lanes_at<N>(R.pc, b);
    }

    /// Blocks some non-halted lane stands at (greedy_groups, ignore_halt).
    static std::uint64_t
    present(const Regs& R)
    {
        std::uint64_t s = 0;
        for(int l = 0; l < N; ++l)
            if(R.pc[l] != HALT) s |= 1ull << R.pc[l];
        return s;
    }

    /// The candidate block with strictly the most lanes, lowest first.
    static int
    major_group(const Regs& R, std::uint64_t set, unsigned& pops)
    {
        int pc = HALT;
        pops   = 0;
        while(set)
        {
            const int      b = std::countr_zero(set);
            const unsigned p = static_cast<unsigned>(std::popcount(lanes_at(R, b)));
            if(p > pops)
            {
                pops = p;
                pc   = b;
            }
            set &= set - 1;
        }
        return pc;
    }

    /// Threaded dispatch from block b, which `pops` lanes stand at: run the
    /// block for its lanes, drop it from the pending set, add every
    /// successor that has lanes, and go on into the successor with the most
    /// lanes (the first in jump-table order on a tie) while that group is
    /// larger than the threshold; returns the pending set.  The kernel's
    /// generated `run_from` does this with its successors compiled into
    /// each block's exit (direct jumps, no tables).
    static std::uint64_t
    dispatch(int b, unsigned pops, Regs& R, std::uint64_t pending, const unsigned threshold, const Ctx& ctx,
             Counters& c)
    {
        return G::run_from(b, pops, R, pending, threshold, ctx, c);
    }

    /// Compact execution of one gang until every lane has halted.
    static void
    compact(Regs& R, const Ctx& ctx, Counters& c)
    {
        if(NB == 0) return;
        const unsigned p0      = static_cast<unsigned>(std::popcount(lanes_at(R, 0)));
        std::uint64_t  pending = p0 ? dispatch(0, p0, R, 0ull, 0u, ctx, c) : 0ull;
        while(present(R))
        {
            unsigned pops = 0;
            int      pc   = major_group(R, pending, pops);
            if(!pops) pc = major_group(R, present(R), pops);
            pending = dispatch(pc, pops, R, pending, 0u, ctx, c);
        }
    }

    /// One chunk of the hybrid visitor with threshold t.
    static void
    hybrid_chunk(Regs& R, const unsigned t, const Ctx& ctx, Counters& c)
    {
        unsigned      pops    = 0;
        int           pc      = major_group(R, present(R), pops);
        std::uint64_t pending = 0;
        while(pops > t)
        {
            pending = dispatch(pc, pops, R, pending, t, ctx, c);
            pops    = 0;
            if(pending) pc = major_group(R, pending, pops);
            if(!pops) pc = major_group(R, present(R), pops);
        }
    }
};

constexpr unsigned long long kNoThread = ~0ull;

/// Shared input cursor of the workers.
struct Cursor
{
    std::atomic<unsigned long long> next{0};
    unsigned long long              n = 0;

    /// Up to k thread indices: [*b, *b + returned).
    unsigned long long
    take(const unsigned long long k, unsigned long long* b)
    {
        if(k == 0) return 0;
        const unsigned long long s = next.fetch_add(k, std::memory_order_relaxed);
        *b                         = s;
        if(s >= n) return 0;
        return s + k <= n ? k : n - s;
    }
};

/// One worker's hybrid stream of `size` threads (Loom's hybrid_stream).
template <typename G>
class Stream
{
    using X                    = Gang<G>;
    static constexpr int    N  = G::N;
    static constexpr int    NB = G::kNumBlocks;
    static constexpr size_t C  = static_cast<size_t>(G::N); // cache-line capacity of the index type

    size_t                     m_size;
    std::vector<unsigned char> m_buf[2];
    typename G::Mem            m_mem[2];
    int                        m_cur = 0;
    size_t                     m_pos = 0; // end of the visited view
    unsigned                   m_gthreshold, m_sthreshold;

    static size_t
    align_up(const size_t x, const size_t a)
    {
        return (x + a - 1) / a * a;
    }

  public:
    typename X::Counters counters;
    std::uint64_t        sorts = 0;

    Stream(const size_t size, const unsigned utr_den) : m_size(align_up(size ? size : C, C))
    {
        for(int i = 0; i < 2; ++i)
        {
            m_buf[i].resize(G::carve_bytes(m_size) + 64);
            auto* base = reinterpret_cast<unsigned char*>(
                (reinterpret_cast<std::uintptr_t>(m_buf[i].data()) + 63) / 64 * 64);
            m_mem[i] = G::carve(base, m_size);
            for(size_t r = 0; r < m_size; ++r)
            {
                m_mem[i].pc[r]  = NB;
                m_mem[i].tid[r] = kNoThread;
            }
        }
        // get_threshold: ceil(x * 1 / den)
        m_gthreshold = static_cast<unsigned>((N + utr_den - 1) / utr_den);
        m_sthreshold = static_cast<unsigned>(align_up((C * NB + utr_den - 1) / utr_den, C));
        m_pos        = m_size;
    }

    const typename G::Mem&
    mem() const
    {
        return m_mem[m_cur];
    }

    size_t
    size() const
    {
        return m_size;
    }

    /// Rows [from, size) take new inputs (or stay empty when none is left),
    /// after the threads they held wrote their outputs.
    void
    exchange(const size_t from, Cursor& cur, const void* const* in, void* const* out)
    {
        const typename G::Mem& m = mem();
        for(size_t r = from; r < m_size; ++r)
            if(m.tid[r] != kNoThread)
            {
                G::finish(m, r, out);
                m.tid[r] = kNoThread;
            }
        unsigned long long b = 0;
        const unsigned long long k = cur.take(m_size - from, &b);
        for(unsigned long long i = 0; i < k; ++i) G::start(m, from + i, in, b + i);
    }

    /// The visitor over the view [0, m_pos).
    void
    visit(const Ctx& ctx)
    {
        const size_t           s = m_pos;
        const unsigned         t = (s > m_sthreshold && s > C) ? m_gthreshold : 0u;
        const typename G::Mem& m = mem();
        typename G::Regs       R;
        for(size_t pos = 0; pos < s && m.pc[pos] != NB; pos += N)
        {
            G::load(R, m, pos);
            X::hybrid_chunk(R, t, ctx, counters);
            G::store(R, m, pos);
        }
    }

    /// Stable counting sort by PC, halted threads last; returns how many
    /// have halted and sets the next view.
    size_t
    sort()
    {
        ++sorts;
        const typename G::Mem& a = m_mem[m_cur];
        const typename G::Mem& b = m_mem[m_cur ^ 1];
        size_t                 bins[NB + 1] = {};
        for(size_t r = 0; r < m_size; ++r) ++bins[a.pc[r]];
        const size_t halted = bins[NB];
        for(int i = 1; i <= NB; ++i) bins[i] += bins[i - 1];
        for(size_t r = m_size; r-- > 0;) G::move(a, r, b, --bins[a.pc[r]]);
        m_cur ^= 1;
        m_pos = halted >= C ? align_up(m_size - halted, C) : m_size;
        return halted;
    }

    /// First row that an exchange may refill (the size when none).
    size_t
    exchange_from() const
    {
        return m_pos;
    }
};

/// The whole job: `threads` workers over threads [0, n).
template <typename G>
int
run(const void* const*  in,
    void* const*        out,
    unsigned long long  n,
    int                 threads,
    const unsigned*     table,
    int                 method,
    unsigned            stream,
    unsigned            utr_den,
    unsigned long long* stats)
{
    if(threads < 1) threads = 1;
    if(utr_den == 0) utr_den = 16;
    if(stream == 0) stream = 288;
    const Cols cols{table};
    const Ctx  ctx{&cols};
    Cursor     cur;
    cur.n = n;
    std::vector<unsigned long long> wstats(static_cast<size_t>(threads) * 3, 0ull);

    auto worker = [&](const int wi)
    {
        using X = Gang<G>;
        typename X::Counters c;
        std::uint64_t        sorts = 0;
        if(method == kCompact)
        {
            // gangs of N consecutive threads, each run to completion
            Stream<G> one(G::N, utr_den); // a gang's worth of rows
            typename G::Regs R;
            for(;;)
            {
                unsigned long long b = 0;
                const unsigned long long k = cur.take(static_cast<unsigned long long>(G::N), &b);
                if(k == 0) break;
                const typename G::Mem& m = one.mem();
                for(int l = 0; l < G::N; ++l)
                {
                    if(static_cast<unsigned long long>(l) < k)
                        G::start(m, static_cast<size_t>(l), in, b + static_cast<unsigned long long>(l));
                    else
                    {
                        m.pc[l]  = G::kNumBlocks;
                        m.tid[l] = kNoThread;
                    }
                }
                G::load(R, m, 0);
                X::compact(R, ctx, c);
                G::store(R, m, 0);
                for(int l = 0; l < G::N; ++l)
                    if(m.tid[l] != kNoThread) G::finish(m, static_cast<size_t>(l), out);
            }
        }
        else
        {
            Stream<G> s(stream, utr_den);
            s.exchange(0, cur, in, out); // set_inputs
            for(;;)
            {
                s.visit(ctx);
                const size_t halted = s.sort();
                // the halted rows past the view: outputs out, inputs in
                if(s.exchange_from() < s.size()) s.exchange(s.exchange_from(), cur, in, out);
                // every row halted and nothing left to take: done
                if(halted == s.size() && s.mem().tid[0] == kNoThread) break;
            }
            c     = s.counters;
            sorts = s.sorts;
        }
        wstats[static_cast<size_t>(wi) * 3 + 0] = c.blocks;
        wstats[static_cast<size_t>(wi) * 3 + 1] = c.lanes;
        wstats[static_cast<size_t>(wi) * 3 + 2] = sorts;
    };

    if(threads == 1)
        worker(0);
    else
    {
        std::vector<std::thread> pool;
        pool.reserve(static_cast<size_t>(threads));
        for(int w = 0; w < threads; ++w) pool.emplace_back(worker, w);
        for(auto& t: pool) t.join();
    }
    if(stats)
    {
        stats[0] = stats[1] = stats[2] = 0;
        for(int w = 0; w < threads; ++w)
            for(int j = 0; j < 3; ++j) stats[j] += wstats[static_cast<size_t>(w) * 3 + j];
    }
    return 0;
}
} // namespace loom_gang
