// Plain drop-in engine: one CUDA thread per Loom thread, in input order.
//
// The generated K::run<> lowers the kernel's basic blocks to a goto CFG
// inside one function, so divergence and reconvergence are the hardware's
// (Blackwell independent thread scheduling).  This replaces Loom's test-only
// CUDA backend (src/vm/cuda.hpp:1329-1579), which launched one kernel per
// basic block and sorted every register column by PC on each round.
#pragma once

#include "common.cuh"

namespace loom_b200
{
/// Launch: grid = ceil(n / blockDim.x), thread tid runs Loom thread tid.
/// Inputs are read once, outputs written once, registers live in CUDA
/// registers; counters[0..1] receive thread/warp VM-instruction totals when
/// kProf is set (lane efficiency = counters[0] / (32 * counters[1])).
template <typename K, bool kProf>
__global__ void
plain_kernel(const Columns                  cols,
             const unsigned long long       n,
             const unsigned long long       max_steps,
             unsigned* __restrict__         status,
             unsigned long long* __restrict__ counters)
{
    const unsigned long long tid =
        static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    Ctx ctx{0ull, max_steps, 0ull, 0ull, status};
    if(tid < n)
    {
        typename K::Regs R;
        K::load_inputs(R, cols, tid);
        K::template run<kProf>(R, ctx);
        K::store_outputs(R, cols, tid);
    }
    if constexpr(kProf)
        flush_counters(counters, ctx.thread_instr, ctx.warp_instr, 0ull);
}

/// Counting hook called at every block entry of K::run<true>.
__device__ __forceinline__ void
count_block(Ctx& ctx, const unsigned n_instr)
{
    const unsigned active = __activemask();
    if((threadIdx.x & 31) == static_cast<unsigned>(__ffs(active) - 1))
        ctx.warp_instr += n_instr;
    ctx.thread_instr += n_instr;
}
} // namespace loom_b200
