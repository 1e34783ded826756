// Regrouping engine: a persistent megakernel that re-forms warps by program
// counter.
//
// Loom's hybrid backend (src/vm/simd.hpp:4024-4292) keeps all thread rows in
// SoA memory, runs aligned chunks predicated while the majority lane count
// stays above the UTR threshold (4163-4194), stores them back, counting-sorts
// every row by PC (2669-2745) and exchanges halted rows for new inputs
// (bve.hpp:1208-1229).  The same method, laid out for Blackwell:
//
//  * state file: one SoA column per register that is live at some block
//    entry, indexed by slot; a parked thread stores only the live-in set of
//    the block it waits at;
//  * per-basic-block work queues of slot ids, double-buffered by round
//    (q[round & 1][block][...]); warps pop 32-entry tiles, so every tile
//    starts with all lanes at one PC;
//  * in registers, a warp keeps executing the block that the largest
//    same-PC lane group stands at (__match_any_sync + __reduce_max_sync)
//    while that group has >= utr lanes and fewer than `period` steps ran;
//  * a halted lane writes its outputs and takes the next input in place
//    (warp-aggregated atomicAdd on the input cursor): the exchange step;
//  * at the end of a tile, lanes are grouped by PC (__match_any_sync), one
//    atomicAdd per group reserves queue space, lanes write their slot ids at
//    base + rank and their live registers to the state file;
//  * rounds are separated by a grid barrier whose wait is bounded; the last
//    CTA to arrive resets the queue counters and decides termination.
// Pure kernels make any execution order valid, so regrouping never changes
// a thread's result (Loom README.md:103-107).
#pragma once

#include "common.cuh"

namespace loom_b200
{
struct RegroupCtl
{
    unsigned           bar_count;
    unsigned           bar_gen;
    unsigned           done;
    unsigned           pad0;
    unsigned long long init_head;    // round-0 admission cursor
    unsigned long long input_cursor; // next input for in-place exchange
};

struct RegroupParams
{
    Columns             cols;
    unsigned*           q;      // [2][num_blocks][cap] slot ids
    unsigned*           qcnt;   // [2][num_blocks]
    unsigned*           qhead;  // [num_blocks] pop cursors of the current round
    unsigned*           tidcol; // [cap] input index of the thread in a slot
    RegroupCtl*         ctl;
    unsigned*           status;
    // accumulated over launches: 0 thread_instr, 1 warp_instr, 2 parks,
    // 3 state bytes, 4 threads finished, 5 rounds
    unsigned long long* counters;
    unsigned long long  n;
    unsigned long long  max_rounds;
    unsigned long long  barrier_spins;
    unsigned            cap;
    unsigned            utr;
    unsigned            period;
    unsigned            refill;
    unsigned            phantoms; // fault injection: CTAs the barrier waits for in vain
};

__device__ __forceinline__ unsigned
ld_volatile(const unsigned* p)
{
    return *reinterpret_cast<const volatile unsigned*>(p);
}

__device__ __forceinline__ unsigned long long
ld_volatile64(const unsigned long long* p)
{
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}

/// Grid barrier with a bounded wait.  The last CTA to arrive runs `last`
/// before releasing the others.  Returns false when the wait ran out (the
/// status word then carries kStatusBarrierTimeout and ctl->done is set).
template <typename F>
__device__ bool
grid_barrier(RegroupCtl*        ctl,
             unsigned*          status,
             unsigned long long spins,
             unsigned           phantoms,
             F&&                last)
{
    __shared__ int ok;
    __syncthreads();
    if(threadIdx.x == 0)
    {
        ok = 1;
        const unsigned gen = ld_volatile(&ctl->bar_gen);
        __threadfence();
        const unsigned arrived = atomicAdd(&ctl->bar_count, 1u);
        if(arrived == gridDim.x - 1 + phantoms)
        {
            last();
            ctl->bar_count = 0;
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        }
        else
        {
            unsigned long long i = 0;
            while(ld_volatile(&ctl->bar_gen) == gen)
            {
                __nanosleep(200);
                if(++i > spins)
                {
                    atomicOr(status, kStatusBarrierTimeout);
                    *reinterpret_cast<volatile unsigned*>(&ctl->done) = 1u;
                    ok = 0;
                    break;
                }
            }
            __threadfence();
        }
    }
    __syncthreads();
    return ok != 0;
}

template <typename K>
__global__ void
regroup_kernel(const RegroupParams p)
{
    constexpr int      B    = K::kNumBlocks;
    constexpr unsigned FULL = 0xffffffffu;

    const unsigned lane  = threadIdx.x & 31u;
    const unsigned gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned long long n_init =
        p.n < static_cast<unsigned long long>(p.cap) ? p.n : p.cap;

    Ctx ctx{0ull, ~0ull, 0ull, 0ull, p.status};
    unsigned long long parks = 0, sbytes = 0, finished = 0;
    typename K::Regs   R;

    for(unsigned round = 0;; ++round)
    {
        const unsigned cur = round & 1u, nxt = cur ^ 1u;
        unsigned       bsel = gwarp % B;

        for(;;)
        {
            // ------------------------------------------------ take a tile
            int                tb = kEmpty;
            unsigned           tk = 0;
            unsigned long long toff = 0;
            if(lane == 0)
            {
                if(round == 0 && ld_volatile64(&p.ctl->init_head) < n_init)
                {
                    const unsigned long long off =
                        atomicAdd(&p.ctl->init_head, 32ull);
                    if(off < n_init)
                    {
                        tb   = kHalt; // marks a fresh-input tile
                        toff = off;
                        tk   = static_cast<unsigned>(
                            n_init - off < 32ull ? n_init - off : 32ull);
                    }
                }
                if(tb == kEmpty)
                    for(int i = 0; i < B; ++i)
                    {
                        const unsigned b   = (bsel + i) % B;
                        const unsigned cnt = ld_volatile(&p.qcnt[cur * B + b]);
                        if(ld_volatile(&p.qhead[b]) >= cnt) continue;
                        const unsigned off = atomicAdd(&p.qhead[b], 32u);
                        if(off < cnt)
                        {
                            tb   = static_cast<int>(b);
                            toff = off;
                            tk   = cnt - off < 32u ? cnt - off : 32u;
                            bsel = b;
                            break;
                        }
                    }
            }
            tb   = __shfl_sync(FULL, tb, 0);
            tk   = __shfl_sync(FULL, tk, 0);
            toff = __shfl_sync(FULL, toff, 0);
            if(tb == kEmpty) break;

            int                pc   = kEmpty;
            unsigned           slot = 0;
            unsigned long long tid  = 0;
            if(lane < tk)
            {
                if(tb == kHalt)
                {
                    slot = static_cast<unsigned>(toff) + lane;
                    tid  = toff + lane;
                    K::load_inputs(R, p.cols, tid);
                    pc = 0;
                }
                else
                {
                    const unsigned long long qi =
                        (static_cast<unsigned long long>(cur) * B + tb) * p.cap +
                        toff + lane;
                    slot = p.q[qi];
                    tid  = p.tidcol[slot];
                    K::restore(tb, R, p.cols, slot);
                    sbytes += K::live_bytes(tb) + 8u;
                    pc = tb;
                }
            }

            // ------------------------------------------------ run
            for(unsigned step = 0;; ++step)
            {
                const unsigned live = __ballot_sync(FULL, pc >= 0);
                if(live == 0u) break;
                const unsigned peers = __match_any_sync(FULL, pc);
                const unsigned key =
                    pc >= 0 ? ((static_cast<unsigned>(__popc(peers)) << 16) |
                               static_cast<unsigned>(pc))
                            : 0u;
                const unsigned best = __reduce_max_sync(FULL, key);
                const int      m    = static_cast<int>(best & 0xffffu);
                const unsigned mc   = best >> 16;
                if(step > 0 && (mc < p.utr || step >= p.period)) break;

                const unsigned ni = K::instr(m);
                if(lane == 0) ctx.warp_instr += ni;
                if(pc == m)
                {
                    ctx.thread_instr += ni;
                    pc = K::exec(m, R, ctx);
                }

                const unsigned hm = __ballot_sync(FULL, pc == kHalt);
                if(hm != 0u)
                {
                    if(pc == kHalt)
                    {
                        K::store_outputs(R, p.cols, tid);
                        ++finished;
                    }
                    if(p.refill)
                    {
                        const int          leader = __ffs(hm) - 1;
                        unsigned long long base   = 0;
                        if(static_cast<int>(lane) == leader)
                            base = atomicAdd(&p.ctl->input_cursor,
                                             static_cast<unsigned long long>(
                                                 __popc(hm)));
                        base = __shfl_sync(FULL, base, leader);
                        if(pc == kHalt)
                        {
                            const unsigned long long t =
                                base + __popc(hm & lanemask_lt());
                            if(t < p.n)
                            {
                                tid = t;
                                K::load_inputs(R, p.cols, t);
                                pc = 0;
                            }
                            else
                                pc = kEmpty;
                        }
                    }
                    else if(pc == kHalt)
                        pc = kEmpty;
                }
            }

            // ------------------------------------------------ park
            const unsigned live = __ballot_sync(FULL, pc >= 0);
            if(pc >= 0)
            {
                const unsigned peers  = __match_any_sync(live, pc);
                const int      leader = __ffs(peers) - 1;
                unsigned       base   = 0;
                if(static_cast<int>(lane) == leader)
                    base = atomicAdd(&p.qcnt[nxt * B + pc],
                                     static_cast<unsigned>(__popc(peers)));
                base = __shfl_sync(peers, base, leader);
                const unsigned idx = base + __popc(peers & lanemask_lt());
                if(idx < p.cap && slot < p.cap)
                {
                    p.q[(static_cast<unsigned long long>(nxt) * B + pc) * p.cap +
                        idx]       = slot;
                    p.tidcol[slot] = static_cast<unsigned>(tid);
                    K::save(pc, R, p.cols, slot);
                    sbytes += K::live_bytes(pc) + 8u;
                    ++parks;
                }
                else
                    ctx.flag(kStatusQueueOverrun);
            }
        }

        // ---------------------------------------------------- round end
        const bool ok = grid_barrier(
            p.ctl,
            p.status,
            p.barrier_spins,
            p.phantoms,
            [&]()
            {
                unsigned long long total = 0;
                for(int b = 0; b < B; ++b)
                {
                    total += ld_volatile(&p.qcnt[nxt * B + b]);
                    p.qcnt[cur * B + b] = 0u;
                    p.qhead[b]          = 0u;
                }
                unsigned done = total == 0ull ? 1u : 0u;
                if(!done && round + 1ull >= p.max_rounds)
                {
                    atomicOr(p.status, kStatusStepLimit);
                    done = 1u;
                }
                *reinterpret_cast<volatile unsigned*>(&p.ctl->done) = done;
                if(done) atomicAdd(p.counters + 5, round + 1ull);
            });
        if(!ok || ld_volatile(&p.ctl->done) != 0u) break;
    }

    flush_counters(p.counters, ctx.thread_instr, ctx.warp_instr, parks);
    flush_counters(p.counters + 3, sbytes, finished, 0ull);
}
} // namespace loom_b200
