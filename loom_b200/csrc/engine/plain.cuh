// Plain drop-in engine: one CUDA thread per Loom thread, in input order.
//
// The generated K::run_burst<> lowers the kernel's basic blocks to a goto CFG
// inside one function, so divergence and reconvergence are the hardware's
// (Blackwell independent thread scheduling).  This replaces Loom's test-only
// CUDA backend (src/vm/cuda.hpp:1329-1579), which launched one kernel per
// basic block and sorted every register column by PC on each round.
#pragma once

#include "common.cuh"

namespace loom_b200
{
/// Launch: grid = ceil(n / blockDim.x), CUDA thread i runs Loom thread
/// first + i (Loom threads [first, first + n); inputs and outputs are
/// indexed by the Loom thread id).  Inputs are read once, outputs written
/// once, registers live in CUDA registers; counters[0..1] receive
/// thread/warp VM-instruction totals when kProf is set (lane efficiency =
/// counters[0] / (32 * counters[1])).
template <typename K, bool kProf>
__global__ void
plain_kernel(const Columns                  cols,
             const unsigned long long       first,
             const unsigned long long       n,
             const unsigned long long       max_steps,
             unsigned* __restrict__         status,
             unsigned long long* __restrict__ counters)
{
    const unsigned long long i =
        static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const unsigned long long tid = first + i;
    __shared__ unsigned long long s_blk[2 * (kProf ? K::kNumBlocks : 1)];
    Ctx ctx{0ull, 0ull, status, &cols, kProf ? s_blk : nullptr};
    if constexpr(kProf) block_counters_clear(s_blk, K::kNumBlocks);
    if(i < n)
    {
        typename K::Regs R;
        K::load_inputs(R, cols, tid);
        // the block budget is the step guard: a thread that has not halted
        // when it runs out is stopped and flagged
        const unsigned budget = max_steps < 0xffffffffull
                                    ? static_cast<unsigned>(max_steps)
                                    : 0xffffffffu;
        if(K::template run_burst<kProf>(0, R, ctx, budget) != kHalt)
            ctx.flag(kStatusStepLimit);
        K::store_outputs(R, cols, tid);
    }
    if constexpr(kProf)
    {
        flush_counters(counters, ctx.thread_instr, ctx.warp_instr, 0ull);
        block_counters_flush(s_blk, K::kNumBlocks, counters + 8);
    }
}

} // namespace loom_b200
