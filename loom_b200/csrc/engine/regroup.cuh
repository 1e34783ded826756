// Regrouping engine: a persistent megakernel that re-forms warps by program
// counter.
//
// Loom's hybrid backend (src/vm/simd.hpp:4024-4292) keeps all thread rows in
// SoA memory, runs aligned chunks predicated while the majority lane count
// stays above the UTR threshold (4163-4194), stores them back, counting-sorts
// every row by PC (2669-2745) and exchanges halted rows for new inputs
// (bve.hpp:1208-1229).  The same method, laid out for Blackwell:
//
//  * per-basic-block work queues that carry the thread state itself: queue
//    (parity, b) is an SoA segment holding, for each waiting thread, the
//    registers live at the entry of block b plus its input index.  Parking a
//    lane group appends contiguous entries (one atomicAdd per group, lanes
//    at base + rank); a tile is 32 consecutive entries, so restores are
//    coalesced loads and every tile starts with all lanes at one PC.  The
//    queues are double-buffered by round parity; the counting sort of the
//    hybrid backend becomes these warp-aggregated appends;
//  * in registers, a warp keeps running the block that the largest same-PC
//    lane group stands at while that group has >= utr lanes and fewer than
//    `period` block steps ran.  A step is a burst of up to `burst` blocks
//    along each lane's own path (hardware reconvergence inside the burst),
//    so the vote costs one ballot per burst; only when the majority block
//    loses its quorum does the warp vote again with __match_any_sync and
//    __reduce_max_sync;
//  * exchange: a halted lane writes its outputs and continues with a new
//    input that it prefetched into registers earlier (one warp-aggregated
//    atomicAdd on the input cursor per claim), so the input load latency is
//    hidden behind the burst;
//  * admission: the input cursor runs against a per-round admission limit
//    that keeps the threads in flight (in lanes or parked) within the
//    population, which bounds every queue;
//  * rounds are separated by a grid barrier whose wait is bounded; the last
//    CTA to arrive resets the queue counters, computes the next admission
//    limit and decides termination.
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
    unsigned long long cursor;     // next input index to admit
    unsigned long long admit_end;  // inputs below this index may enter this round
    unsigned long long next_round; // round number the next launch continues with
    unsigned long long t_first;    // %globaltimer (ns) when the first CTA started
    unsigned long long t_last;     // %globaltimer when the launch finished
};

__device__ __forceinline__ unsigned long long
global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct RegroupParams
{
    Columns             cols;     // inputs then outputs
    char*               state;    // queues with their state: [2][K::kRowBytes * cap]
    unsigned*           qcnt;     // [2][num_blocks] entries per queue
    unsigned*           qhead;    // [num_blocks] pop cursors of the current round
    RegroupCtl*         ctl;
    unsigned*           status;
    // accumulated over launches: 0 thread_instr, 1 warp_instr, 2 parks,
    // 3 state bytes, 4 threads finished, 5 rounds; profiled launches also
    // add thread / warp instructions of block b to 8 + 2b / 9 + 2b
    unsigned long long* counters;
    unsigned long long  n;
    unsigned long long  max_rounds;
    unsigned long long  barrier_spins;
    unsigned            cap;      // population: entries per queue, multiple of 32
    unsigned            utr;      // majority quorum, lanes
    unsigned            period;   // block steps per tile per round (LOOM_B200_PERIOD_UNBOUNDED: none)
    unsigned            burst;    // blocks a lane runs between two votes
    unsigned            spread;   // majority size from which all live lanes run
    unsigned            prefetch; // prefetch the next input of every lane
    unsigned            refill;   // halted lanes claim new inputs at once
    unsigned            phantoms; // fault injection: CTAs the barrier waits for in vain
    // Serving: a launch may run a slice of `slice_rounds` rounds (0: until
    // done) starting at round `round0`, whose parity selects the queues it
    // resumes from; a finished thread adds one to inst_done[its instance id]
    // (NULL: no per-instance counts).
    unsigned            round0;
    unsigned            slice_rounds;
    unsigned*           inst_done;
    // Cost model: a block's quorum is the larger of utr and K::quorum(b),
    // and blocks with a quorum are entered only at the start of a burst.
    unsigned            cost_model;
    // Warp schedule: 0 runs the largest group that meets its quorum; 1 runs
    // the group at the block earliest in reverse post-order, so lanes that
    // lag catch up with the others and merge at join blocks and loop heads;
    // 2 steps one block at a time in that order with no vote and no quorum
    // (lanes park only when the period ends); 3 runs every live lane along
    // its own path under the hardware's reconvergence, as the plain engine
    // does, and takes new threads for the whole warp once all its lanes have
    // finished (for kernels whose lanes the hardware keeps together).
    unsigned            schedule;
    // Schedule 2: a long block (K::long_block) runs only once this many of
    // the warp's lanes stand at it, or when no other block is left (0: off).
    unsigned            defer_lanes;
    // Schedule 2, kernels with one call site (K::kSplitCallSites false):
    // iterations of a self-loop a lane runs within one step before the step
    // ends at the loop's header (0: kSelfLoopSpin; small kernels run 16, 64
    // or kSelfLoopSpin, constants their tight loops are compiled with: up to
    // 16, up to 64, more).
    unsigned            spin_iters;
    // Schedule 2: a burst ends once this many of the warp's lanes have
    // halted (their replacements then start together; 0: full bursts).
    unsigned            refill_lanes;
    // Full tiles come back through shared memory: one bulk copy (TMA,
    // cp.async.bulk) per slot column of the tile, then each lane reads its
    // entry there (the launch's dynamic shared memory holds a staging area
    // and an mbarrier per warp); 0 restores with 128-bit loads from HBM.
    unsigned            bulk_restore;
};

/// Dynamic shared memory of a launch with bulk_restore: an mbarrier per warp
/// (16-byte aligned block), then 32 entries of the largest queue row per warp.
__host__ __device__ constexpr unsigned
bulk_stage_bytes(const unsigned warps, const unsigned max_stage_row)
{
    return (warps * 8u + 15u) / 16u * 16u + warps * 32u * max_stage_row;
}

/// Iterations of a self-loop a lane runs within one step of schedule 2
/// before the step ends at the loop's header (opts.spin_iters: 0).
constexpr unsigned kSelfLoopSpin = 1024;

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

/// Grid barrier with a bounded wait.  The first warp of the last CTA to
/// arrive runs `last` (every lane of it: the round-end work is spread over
/// the warp) before releasing the others.  Returns whether the CTA should
/// run another round: false when the launch is done or when the wait ran
/// out (the status word then carries kStatusBarrierTimeout and ctl->done is
/// set).  The value is decided by thread 0 and shared, so every thread of
/// the CTA leaves the round loop together.
template <typename F>
__device__ bool
grid_barrier(RegroupCtl*        ctl,
             unsigned*          status,
             unsigned long long spins,
             unsigned           phantoms,
             bool               final_round,
             F&&                last)
{
    __shared__ int      ok;
    __shared__ int      is_last;
    __shared__ unsigned gen0;
    __syncthreads();
    if(threadIdx.x == 0)
    {
        gen0 = ld_volatile(&ctl->bar_gen);
        __threadfence();
        const unsigned arrived = atomicAdd(&ctl->bar_count, 1u);
        is_last = arrived == gridDim.x - 1 + phantoms ? 1 : 0;
    }
    __syncthreads();
    if(is_last)
    {
        if(threadIdx.x < 32)
        {
            __threadfence();
            last();
            __threadfence(); // every lane's resets visible before the release
            __syncwarp();
            if(threadIdx.x == 0)
            {
                ctl->bar_count = 0;
                __threadfence();
                atomicAdd(&ctl->bar_gen, 1u);
                ok = ld_volatile(&ctl->done) != 0u ? 0 : 1;
            }
        }
        __syncthreads();
        return ok != 0;
    }
    if(threadIdx.x == 0)
    {
        int            go  = 1;
        const unsigned gen = gen0;
        if(final_round)
        {
            // the launch ends with this round whatever the last CTA finds:
            // nothing to wait for (the CTAs need not be resident together)
            go = 0;
        }
        else
        {
            unsigned long long i = 0;
            while(ld_volatile(&ctl->bar_gen) == gen)
            {
                __nanosleep(100);
                if(++i > spins)
                {
                    atomicOr(status, kStatusBarrierTimeout);
                    *reinterpret_cast<volatile unsigned*>(&ctl->done) = 1u;
                    go = 0;
                    break;
                }
            }
            __threadfence();
        }
        if(ld_volatile(&ctl->done) != 0u) go = 0;
        ok = go;
    }
    __syncthreads();
    return ok != 0;
}

/// Claims input indices for the lanes in `need` with one atomicAdd for the
/// warp.  Returns this lane's index, or ~0 when the lane got none; `dry`
/// turns true once the round's admission limit is reached.
__device__ __forceinline__ unsigned long long
claim_inputs(const unsigned need, RegroupCtl* ctl, unsigned long long admit_end, bool& dry)
{
    constexpr unsigned FULL   = 0xffffffffu;
    const unsigned     lane   = threadIdx.x & 31u;
    const int          leader = __ffs(need) - 1;
    unsigned long long base   = 0;
    if(static_cast<int>(lane) == leader)
        base = atomicAdd(&ctl->cursor, static_cast<unsigned long long>(__popc(need)));
    base = __shfl_sync(FULL, base, leader);
    if(base + __popc(need) >= admit_end) dry = true;
    const unsigned long long t = base + __popc(need & lanemask_lt());
    return ((need >> lane) & 1u) && t < admit_end ? t : ~0ull;
}

/// The megakernel.  `__maxnreg__` holds it to a register cap (`kRegs`, by
/// default `K::kRegroupMaxRegs`) so that enough warps stay resident to hide
/// the latency of the lanes it keeps running; `kBulk` compiles the staged
/// (bulk-copy) tile restore in.  With `kPark` false the kernel serves only
/// launches that never park (schedule 2 or 3, no period) and do not
/// prefetch: it has no queue pop, restore or park code, no group selection
/// of schedules 0 and 1 and no input prefetch, code that such launches never
/// run but that would still cost registers.
template <typename K, bool kProf, int kRegs = K::kRegroupMaxRegs, bool kBulk = false, bool kPark = true>
__global__ void __maxnreg__(kRegs)
regroup_kernel(const RegroupParams p)
{
    constexpr int      B    = K::kNumQueues;
    constexpr unsigned FULL = 0xffffffffu;
    const unsigned lane  = threadIdx.x & 31u;
    const unsigned gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    __shared__ unsigned long long s_blk[2 * (kProf ? K::kNumBlocks : 1)];
    Ctx ctx{0ull, 0ull, p.status, &p.cols, kProf ? s_blk : nullptr};
    if constexpr(kProf) block_counters_clear(s_blk, K::kNumBlocks);
    // block ranks in reverse post-order, for the schedules that order groups
    __shared__ unsigned s_rank[K::kNumBlocks];
    for(int i = threadIdx.x; i < K::kNumBlocks; i += blockDim.x) s_rank[i] = K::rank(i);
    if(threadIdx.x == 0) atomicMin(&p.ctl->t_first, global_ns());
    __syncthreads();
    // per-lane counters, 32 bits (a lane's share of one launch), summed into
    // the 64-bit launch counters at the end
    unsigned           parks = 0, sbytes = 0, finished = 0;
    // the round's admission limit, read once per CTA
    __shared__ unsigned long long s_admit_end;
    typename K::Regs   R;
    typename K::In     pf;
    unsigned long long pf_tid = ~0ull;
    const bool         cost_on = p.cost_model != 0u;
    // staged restore: this warp's mbarrier and staging area
    extern __shared__ __align__(16) unsigned char s_dyn[];
    const unsigned      wib   = threadIdx.x >> 5;
    unsigned long long* mbar  = reinterpret_cast<unsigned long long*>(s_dyn) + wib;
    unsigned char*      stage = s_dyn + (blockDim.x / 32u * 8u + 15u) / 16u * 16u + wib * 32u * K::kMaxStageRow;
    // the staged restore is compiled into its own instantiation (kBulk):
    // its code would cost the other launches registers
    bool                bulk_ok    = kBulk && p.bulk_restore != 0u;
    unsigned            bulk_phase = 0;
    if(bulk_ok)
    {
        if(lane == 0) mbar_init(mbar);
        __syncwarp();
    }
    // lanes a group at block b needs to keep running
    auto need = [&](const int b) -> unsigned
    {
        const unsigned q = cost_on ? K::quorum(b) : 0u;
        return q > p.utr ? q : p.utr;
    };
    for(unsigned round = p.round0;; ++round)
    {
        const unsigned           cur = round & 1u, nxt = cur ^ 1u;
        if(threadIdx.x == 0) s_admit_end = ld_volatile64(&p.ctl->admit_end);
        __syncthreads();
        const unsigned long long& admit_end = s_admit_end;
        unsigned                 bsel = gwarp % B;
        bool                     dry  = false;
        for(;;)
        {
            // a tile of the current round's queues: the warp reads 32
            // queues' counts and pop cursors at once, and takes 32 entries
            // from the first non-empty queue at or after bsel (warps start
            // at different queues, so they contend less)
            int      tb = kEmpty;
            unsigned tk = 0, toff = 0;
            for(int c = 0; kPark && c < (B + 31) / 32 && tb < 0; ++c)
            {
                const int base = ((static_cast<int>(bsel) / 32 + c) % ((B + 31) / 32)) * 32;
                const int b    = base + static_cast<int>(lane);
                unsigned  cnt  = 0, head = 0;
                if(b < B)
                {
                    cnt  = ld_volatile(&p.qcnt[cur * B + b]);
                    cnt  = cnt > p.cap ? p.cap : cnt;
                    head = ld_volatile(&p.qhead[b]);
                }
                unsigned avail = __ballot_sync(FULL, b < B && head < cnt);
                const unsigned s0 = c == 0 ? bsel % 32u : 0u;
                while(avail)
                {
                    // first available queue at or after s0, cyclically
                    const unsigned rot  = s0 ? ((avail >> s0) | (avail << (32u - s0))) : avail;
                    const unsigned pick = (static_cast<unsigned>(__ffs(rot)) - 1u + s0) & 31u;
                    unsigned       off  = 0;
                    if(lane == pick) off = atomicAdd(&p.qhead[b], 32u);
                    off                = __shfl_sync(FULL, off, static_cast<int>(pick));
                    const unsigned pc_ = __shfl_sync(FULL, cnt, static_cast<int>(pick));
                    if(off < pc_)
                    {
                        tb   = base + static_cast<int>(pick);
                        toff = off;
                        tk   = pc_ - off < 32u ? pc_ - off : 32u;
                        bsel = static_cast<unsigned>(tb);
                        break;
                    }
                    avail &= ~(1u << pick);
                }
            }
            int                pc  = kEmpty;
            unsigned long long tid = 0;
            if(kPark && tb >= 0)
            {
                bool staged = false;
                if(bulk_ok && tk == 32u)
                {
                    // the tile through shared memory: lane 0 issues a bulk
                    // copy per slot column, every lane waits (bounded) for
                    // the mbarrier's phase
                    bool issued = false;
                    __syncwarp(); // the lanes' reads of the previous tile are done
                    if(lane == 0)
                    {
                        // order those generic-proxy reads before the bulk
                        // copies' writes to the same shared memory
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        issued = K::bulk_issue(tb, stage, p.state + static_cast<unsigned long long>(cur) * K::kRowBytes * p.cap,
                                               p.cap, toff, mbar);
                    }
                    issued = __shfl_sync(FULL, issued ? 1u : 0u, 0) != 0u;
                    if(issued)
                    {
                        bool     done = false;
                        unsigned i    = 0;
                        while(!(done = mbar_try_wait(mbar, bulk_phase)) && ++i < (1u << 20)) {}
                        if(__all_sync(FULL, done))
                        {
                            bulk_phase ^= 1u;
                            staged = true;
                        }
                        else
                        {
                            // the copy did not complete in time: restore from
                            // HBM, and stage no more tiles in this launch
                            ctx.flag(kStatusBarrierTimeout);
                            bulk_ok = false;
                        }
                    }
                    __syncwarp();
                }
                if(lane < tk)
                {
                    // the queue keeps the low 32 bits of the thread id
                    const unsigned t32 = staged ? K::restore_stage(tb, R, stage, lane)
                                                : K::restore(tb, R, p.state, p.cap, cur, toff + lane);
                    tid = p.cols.tid_base + static_cast<unsigned>(t32 - static_cast<unsigned>(p.cols.tid_base));
                    if(tid < p.n) { pc = K::block_of(tb); sbytes += K::live_bytes(tb) + 4u; }
                    else ctx.flag(kStatusQueueOverrun);
                }
                tb = K::block_of(tb);
            }
            else
            {
                if(dry) break;
                const unsigned long long t = claim_inputs(FULL, p.ctl, admit_end, dry);
                if(__ballot_sync(FULL, t != ~0ull) == 0u) break;
                if(t != ~0ull) { typename K::In in; K::load_in(in, p.cols, t); K::start(R, in); tid = t; pc = 0; }
                tb = 0; tk = 32u;
            }
            int      m     = tb;
            unsigned mc    = tk;
            unsigned steps = 0;
            for(;;)
            {
                if(kPark && p.prefetch && !dry)
                {
                    const unsigned need = __ballot_sync(FULL, pf_tid == ~0ull);
                    if(need)
                    {
                        const unsigned long long t = claim_inputs(need, p.ctl, admit_end, dry);
                        if(t != ~0ull) { pf_tid = t; K::load_in(pf, p.cols, t); }
                    }
                }
                // Schedule 2 steps one loop iteration at a time, always the
                // block earliest in reverse post-order among the warp's lanes:
                // lanes that lag run until they reach the others (MinPC
                // stepping, the order a reconvergence stack keeps); a long
                // block waits until defer_lanes lanes stand at it or no
                // other block is left.  Schedule 3 runs every live lane
                // along its own path, the hardware reconverging the warp as
                // in the plain engine; schedules 0 and 1 run the chosen group
                // (or every live lane once the group has spread_lanes).
                // Large kernels keep one copy of their code in the megakernel
                // (one call site, the spin count a runtime value); small ones
                // get a call site per kind of step, so that a tight
                // self-loop is compiled with its spin count known.
                const bool minpc = p.schedule == 2u;
                for(unsigned i = 0; i < (minpc ? p.burst : 1u); ++i)
                {
                    bool run;
                    if(minpc)
                    {
                        unsigned rk = pc >= 0 ? s_rank[pc] : 0xffffffffu;
                        if(p.defer_lanes)
                            for(int j = 0; j < K::kNumLong; ++j)
                            {
                                const int      h  = K::long_block(j);
                                const unsigned at = __ballot_sync(FULL, pc == h);
                                if(pc == h && static_cast<unsigned>(__popc(at)) < p.defer_lanes) rk |= 0x10000u;
                            }
                        const unsigned lo = __reduce_min_sync(FULL, rk);
                        if(lo == 0xffffffffu) break;
                        run = rk == lo;
                    }
                    else
                        run = pc >= 0 && (p.schedule == 3u || mc >= p.spread || pc == m);
                    if(run)
                    {
                        if constexpr(K::kSplitCallSites)
                        {
                            // a self-loop's spin count is compiled into each
                            // call site: spin_iters picks 16, 64 or the
                            // default (a few iterations let halted lanes take
                            // new threads while the others keep looping)
                            if(minpc && p.spin_iters && p.spin_iters <= 16u)
                                pc = K::template run_burst<kProf>(pc, R, ctx, 1u, false, 16u);
                            else if(minpc && p.spin_iters && p.spin_iters <= 64u)
                                pc = K::template run_burst<kProf>(pc, R, ctx, 1u, false, 64u);
                            else if(minpc)
                                pc = K::template run_burst<kProf>(pc, R, ctx, 1u, false, kSelfLoopSpin);
                            else
                                pc = K::template run_burst<kProf>(pc, R, ctx, p.burst, kPark && cost_on && p.schedule < 2u);
                        }
                        else
                            pc = K::template run_burst<kProf>(pc, R, ctx, minpc ? 1u : p.burst,
                                                              kPark && cost_on && p.schedule < 2u,
                                                              minpc ? (p.spin_iters ? p.spin_iters : kSelfLoopSpin) : 0u);
                    }
                    if(minpc && p.refill_lanes &&
                       static_cast<unsigned>(__popc(__ballot_sync(FULL, pc == kHalt))) >= p.refill_lanes)
                        break;
                }
                if(kPark && p.period != LOOM_B200_PERIOD_UNBOUNDED) steps += p.burst;
                const unsigned hm = __ballot_sync(FULL, pc == kHalt);
                if(hm != 0u)
                {
                    if(pc == kHalt)
                    {
                        K::store_outputs(R, p.cols, tid);
                        ++finished;
                        if(p.inst_done)
                        {
                            // one atomic per instance among the halting lanes
                            const unsigned id    = instance_id(p.cols, tid);
                            const unsigned peers = __match_any_sync(hm, id);
                            if(static_cast<int>(lane) == __ffs(peers) - 1)
                                atomicAdd(p.inst_done + id, static_cast<unsigned>(__popc(peers)));
                        }
                        pc = kEmpty;
                        if(pf_tid != ~0ull && p.schedule != 3u) { K::start(R, pf); tid = pf_tid; pf_tid = ~0ull; pc = 0; }
                    }
                    if(!dry && p.refill && p.schedule != 3u)
                    {
                        const unsigned need = __ballot_sync(FULL, pc == kEmpty);
                        if(need)
                        {
                            const unsigned long long t = claim_inputs(need, p.ctl, admit_end, dry);
                            if(t != ~0ull) { typename K::In in; K::load_in(in, p.cols, t); K::start(R, in); tid = t; pc = 0; }
                        }
                    }
                }
                if(kPark && steps >= p.period) break;
                if(p.schedule == 3u)
                {
                    // the warp takes new threads only when all its lanes
                    // have finished, so that they start together at block 0
                    // (the plain engine's lockstep, one warp of threads
                    // after another)
                    if(__ballot_sync(FULL, pc >= 0) != 0u) continue;
                    if(pf_tid != ~0ull) { K::start(R, pf); tid = pf_tid; pf_tid = ~0ull; pc = 0; }
                    const unsigned need = __ballot_sync(FULL, pc == kEmpty);
                    if(need && !dry)
                    {
                        const unsigned long long t = claim_inputs(need, p.ctl, admit_end, dry);
                        if(t != ~0ull) { typename K::In in; K::load_in(in, p.cols, t); K::start(R, in); tid = t; pc = 0; }
                    }
                    if(__ballot_sync(FULL, pc >= 0) == 0u) break;
                    continue;
                }
                if(p.schedule == 2u)
                {
                    // a lane left empty by a refill that found no input
                    // takes its prefetched one, so a warp leaves the loop
                    // with no input claimed and none parked
                    if(pc == kEmpty && pf_tid != ~0ull) { K::start(R, pf); tid = pf_tid; pf_tid = ~0ull; pc = 0; }
                    // no quorum: the warp keeps its lanes until the period
                    // ends or none is left
                    if(__ballot_sync(FULL, pc >= 0) == 0u) break;
                    continue;
                }
                if constexpr(!kPark) break; // schedules 0 and 1 always park
                const unsigned cm = __popc(__ballot_sync(FULL, pc == m));
                if(!p.schedule && cm >= need(m)) { mc = cm; continue; }
                // the group to run next among those that meet their block's
                // quorum: the largest, or the one earliest in program order
                const unsigned peers = __match_any_sync(FULL, pc);
                const unsigned gs    = static_cast<unsigned>(__popc(peers));
                const bool     elig  = pc >= 0 && gs >= need(pc);
                const unsigned prio  = p.schedule ? 0xffffu - K::rank(pc) : gs;
                const unsigned key   = elig ? ((prio << 16) | static_cast<unsigned>(pc)) : 0u;
                const unsigned best  = __reduce_max_sync(FULL, key);
                if(best == 0u) break;
                m  = static_cast<int>(best & 0xffffu);
                mc = p.schedule ? static_cast<unsigned>(__popc(__ballot_sync(FULL, pc == m))) : best >> 16;
            }
            if constexpr(!kPark)
            {
                // nothing to park: a lane still live here means the launch
                // was not one that never parks
                if(pc >= 0 || pf_tid != ~0ull) ctx.flag(kStatusQueueOverrun);
                continue;
            }
            for(int pass = 0; pass < 2; ++pass)
            {
                if(pass == 1)
                {
                    if(__ballot_sync(FULL, pf_tid != ~0ull) == 0u) break;
                    pc = kEmpty;
                    if(pf_tid != ~0ull) { K::start(R, pf); tid = pf_tid; pf_tid = ~0ull; pc = 0; }
                }
                const unsigned live = __ballot_sync(FULL, pc >= 0);
                if(pc >= 0)
                {
                    const int      q      = K::queue_of(pc, R);
                    const unsigned peers  = __match_any_sync(live, q);
                    const int      leader = __ffs(peers) - 1;
                    unsigned       base   = 0;
                    if(static_cast<int>(lane) == leader)
                        base = atomicAdd(&p.qcnt[nxt * B + q], static_cast<unsigned>(__popc(peers)));
                    base = __shfl_sync(peers, base, leader);
                    const unsigned idx = base + __popc(peers & lanemask_lt());
                    if(idx < p.cap)
                    {
                        K::save(q, R, p.state, p.cap, nxt, idx, static_cast<unsigned>(tid));
                        sbytes += K::live_bytes(q) + 4u;
                        ++parks;
                    }
                    else ctx.flag(kStatusQueueOverrun);
                }
            }
        }

        // ---------------------------------------------------- round end
        const bool more = grid_barrier(
            p.ctl,
            p.status,
            p.barrier_spins,
            p.phantoms,
            p.slice_rounds == 1u,
            [&]()
            {
                // every lane of the first warp of the last CTA: the threads
                // parked for the next round (summed over the queues), the
                // current round's counts and pop cursors cleared; lane 0
                // then sets the next admission limit and decides the end
                unsigned long long parked = 0;
                for(int b = static_cast<int>(lane); b < B; b += 32)
                {
                    parked += ld_volatile(&p.qcnt[nxt * B + b]);
                    p.qcnt[cur * B + b] = 0u;
                    p.qhead[b]          = 0u;
                }
                for(int o = 16; o > 0; o >>= 1) parked += __shfl_xor_sync(FULL, parked, o);
                if(lane != 0) return;
                // claims beyond the limit were refused: give them back
                unsigned long long c = ld_volatile64(&p.ctl->cursor);
                if(c > admit_end) c = admit_end;
                const unsigned long long room = parked < p.cap ? p.cap - parked : 0ull;
                p.ctl->cursor    = c;
                p.ctl->admit_end = c + room < p.n ? c + room : p.n;
                unsigned done    = parked == 0ull && c >= p.n ? 1u : 0u;
                const unsigned long long ran = round + 1ull - p.round0;
                if(!done && p.slice_rounds && ran >= p.slice_rounds)
                    done = 1u; // end of the slice: the parked threads wait for the next one
                else if(!done && ran >= p.max_rounds)
                {
                    atomicOr(p.status, kStatusStepLimit);
                    done = 1u;
                }
                p.ctl->next_round = round + 1ull;
                if(done) p.ctl->t_last = global_ns();
                *reinterpret_cast<volatile unsigned*>(&p.ctl->done) = done;
                if(done) atomicAdd(p.counters + 5, ran);
            });
        if(!more) break;
    }

    flush_counters(p.counters, ctx.thread_instr, ctx.warp_instr, static_cast<unsigned long long>(parks));
    flush_counters(p.counters + 3, static_cast<unsigned long long>(sbytes), static_cast<unsigned long long>(finished), 0ull);
    if constexpr(kProf) block_counters_flush(s_blk, K::kNumBlocks, p.counters + 8);
}
} // namespace loom_b200
