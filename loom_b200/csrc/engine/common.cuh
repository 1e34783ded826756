// Shared device-side definitions of the B200 Loom engine.
//
// Generated kernel code (loom_b200/csrc/gen/*.cu) includes this header; the
// engines in plain.cuh and regroup.cuh are templates over the generated
// kernel structs.
#pragma once

#include <cstdint>
#include <cstring>

#include "loom_b200.h"

namespace loom_b200
{
/// Maximum number of columns (inputs + outputs) per kernel; the pointer
/// table travels in the kernel's parameter space.
constexpr int kMaxCols = 64;
/// Maximum number of input columns.
constexpr int kMaxIn = 16;

/// Block index used for "thread finished" (Loom's halt_pos, core.hpp:985).
constexpr int kHalt = -1;
/// Lane holds no thread.
constexpr int kEmpty = -2;

/// Input and output columns of a launch, plus what the input forms and the
/// table op read.  Input i is read according to form[i]
/// (LOOM_B200_IN_*): an array, the thread index, a broadcast value, the
/// thread index within its instance, or the instance index.
struct Columns
{
    void*                     p[kMaxCols];
    unsigned                  form[kMaxIn];
    unsigned long long        value[kMaxIn];
    const unsigned long long* inst_start; // num_inst + 1 thread offsets
    unsigned                  num_inst;
    const unsigned*           table;      // words read by the tab op
    // Serving: array columns are rings indexed by tid & ring_mask (0: by
    // tid); the instance form reads inst_id[i] (NULL: i); every thread id in
    // flight lies in [tid_base, tid_base + 2^32), so the 32-bit ids kept in
    // the queue state name one thread each.
    unsigned long long        ring_mask;
    unsigned long long        tid_base;
    const unsigned*           inst_id;
};

/// Position of thread `tid` in the array columns.
__device__ __forceinline__ unsigned long long
col_index(const Columns& c, const unsigned long long tid)
{
    return c.ring_mask ? (tid & c.ring_mask) : tid;
}

/// Status bits written by device code (also returned through the C ABI).
enum : unsigned
{
    kStatusStepLimit    = LOOM_B200_STATUS_STEP_LIMIT,
    kStatusAssertFp     = LOOM_B200_STATUS_ASSERT_FP,
    kStatusQueueOverrun = LOOM_B200_STATUS_QUEUE_OVERRUN,
    kStatusBarrierTimeout = LOOM_B200_STATUS_BARRIER_TIMEOUT,
};

struct Columns;

/// Per-thread execution context: instruction counters, the status word and
/// the launch's columns (for the table op).
struct Ctx
{
    unsigned long long thread_instr;
    unsigned long long warp_instr;
    unsigned*          status;
    const Columns*     cols;
    unsigned long long* blk; // profiled launches: per-block counters in shared memory

    __device__ __forceinline__ void
    flag(unsigned bit)
    {
        atomicOr(status, bit);
    }
};

template <typename To, typename From>
__device__ __forceinline__ To
bitcast(const From v)
{
    static_assert(sizeof(To) == sizeof(From), "bitcast needs equal sizes");
    To r;
    memcpy(&r, &v, sizeof(To));
    return r;
}

// C++ library semantics of the Loom op set (Loom src/vm/operators.hpp).
// std::max / std::min: (a < b) ? b : a and (b < a) ? b : a.
template <typename T>
__device__ __forceinline__ T
op_max(const T a, const T b)
{
    return (a < b) ? b : a;
}
template <typename T>
__device__ __forceinline__ T
op_min(const T a, const T b)
{
    return (b < a) ? b : a;
}

__device__ __forceinline__ float op_abs(float v) { return fabsf(v); }
__device__ __forceinline__ double op_abs(double v) { return fabs(v); }
__device__ __forceinline__ int op_abs(int v) { return v < 0 ? -v : v; }
__device__ __forceinline__ long long op_abs(long long v) { return v < 0 ? -v : v; }

__device__ __forceinline__ float op_round(float v) { return roundf(v); }
__device__ __forceinline__ double op_round(double v) { return round(v); }
__device__ __forceinline__ float op_ceil(float v) { return ceilf(v); }
__device__ __forceinline__ double op_ceil(double v) { return ceil(v); }
__device__ __forceinline__ float op_floor(float v) { return floorf(v); }
__device__ __forceinline__ double op_floor(double v) { return floor(v); }
__device__ __forceinline__ float op_trunc(float v) { return truncf(v); }
__device__ __forceinline__ double op_trunc(double v) { return trunc(v); }
__device__ __forceinline__ float op_sqrt(float v) { return sqrtf(v); }
__device__ __forceinline__ double op_sqrt(double v) { return sqrt(v); }
// Float sin and cos are evaluated in double and rounded once to float: the
// result is the correctly rounded value except within a hair of a rounding
// boundary, which is what the host's libm (the scalar backend's std::sin,
// operators.hpp:314-325) returns for all but a few arguments.
__device__ __forceinline__ float op_sin(float v) { return static_cast<float>(sin(static_cast<double>(v))); }
__device__ __forceinline__ double op_sin(double v) { return sin(v); }
__device__ __forceinline__ float op_cos(float v) { return static_cast<float>(cos(static_cast<double>(v))); }
__device__ __forceinline__ double op_cos(double v) { return cos(v); }
__device__ __forceinline__ float op_copysign(float a, float b) { return copysignf(a, b); }
__device__ __forceinline__ double op_copysign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ float op_fma(float x, float y, float z) { return fmaf(x, y, z); }
__device__ __forceinline__ double op_fma(double x, double y, double z) { return fma(x, y, z); }
// rsqrt is 1 / sqrt(x) with IEEE division and square root (operators.hpp:166-174).
__device__ __forceinline__ float op_rsqrt(float v) { return 1.0f / sqrtf(v); }
__device__ __forceinline__ double op_rsqrt(double v) { return 1.0 / sqrt(v); }

/// assert_fp (operators.hpp:256-276) aborts the host process on NaN or
/// infinity; on the device it raises a status bit and passes the value on.
template <typename T>
__device__ __forceinline__ T
op_assert_fp(const T v, Ctx& ctx)
{
    if(!isfinite(v)) ctx.flag(kStatusAssertFp);
    return v;
}

__device__ __forceinline__ unsigned
lanemask_lt()
{
    unsigned m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

/// Counting hook at every block entry of K::run_burst<true>: the lowest
/// active lane adds the block's instruction count once for the warp, every
/// lane adds it for itself (lane efficiency = thread / (32 * warp)).
/// With a per-block array (profiled launches), the lowest lane also adds
/// the block's thread and warp instructions to entry 2b and 2b + 1 there.
__device__ __forceinline__ void
count_block(Ctx& ctx, const int b, const unsigned n_instr)
{
    const unsigned active = __activemask();
    if((threadIdx.x & 31) == static_cast<unsigned>(__ffs(active) - 1))
    {
        ctx.warp_instr += n_instr;
        if(ctx.blk)
        {
            atomicAdd(ctx.blk + 2 * b, static_cast<unsigned long long>(__popc(active)) * n_instr);
            atomicAdd(ctx.blk + 2 * b + 1, static_cast<unsigned long long>(n_instr));
        }
    }
    ctx.thread_instr += n_instr;
}

/// Shared per-block counters of a profiled launch: cleared at kernel start,
/// added into dst[0 .. 2 * nb) at the end (every thread of the CTA calls both).
__device__ __forceinline__ void
block_counters_clear(unsigned long long* s, const int nb)
{
    for(int i = threadIdx.x; i < 2 * nb; i += blockDim.x) s[i] = 0ull;
    __syncthreads();
}

__device__ __forceinline__ void
block_counters_flush(const unsigned long long* s, const int nb, unsigned long long* dst)
{
    __syncthreads();
    for(int i = threadIdx.x; i < 2 * nb; i += blockDim.x)
        if(s[i]) atomicAdd(dst + i, s[i]);
}

/// Instance of thread `tid`: the last i with inst_start[i] <= tid.
__device__ __forceinline__ unsigned
find_instance(const Columns& c, const unsigned long long tid)
{
    unsigned lo = 0, hi = c.num_inst; // inst_start[lo] <= tid < inst_start[hi]
    while(hi - lo > 1)
    {
        const unsigned mid = (lo + hi) >> 1;
        if(c.inst_start[mid] <= tid)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

/// Instance id of thread `tid`: its position among the instances, or the
/// id that inst_id gives that position.
__device__ __forceinline__ unsigned
instance_id(const Columns& c, const unsigned long long tid)
{
    if(!c.num_inst) return 0u;
    const unsigned i = find_instance(c, tid);
    return c.inst_id ? c.inst_id[i] : i;
}

/// Input i of thread `tid` as T.
template <typename T>
__device__ __forceinline__ T
load_input(const Columns& c, const int i, const unsigned long long tid)
{
    switch(c.form[i])
    {
    case LOOM_B200_IN_ARRAY: return static_cast<const T*>(c.p[i])[col_index(c, tid)];
    case LOOM_B200_IN_BROADCAST:
    {
        T v;
        memcpy(&v, &c.value[i], sizeof(T));
        return v;
    }
    case LOOM_B200_IN_LOCAL_IOTA:
        return static_cast<T>(c.num_inst ? tid - c.inst_start[find_instance(c, tid)] : tid);
    case LOOM_B200_IN_INSTANCE: return static_cast<T>(instance_id(c, tid));
    default: return static_cast<T>(tid);
    }
}

/// The tab op (a Loom extension): word `idx` of the launch's table as T,
/// through the read-only data path.
template <typename T>
__device__ __forceinline__ T
table_load(const Columns& c, const unsigned idx)
{
    return bitcast<T>(__ldg(c.table + idx));
}

// ---- bulk copies (TMA, untiled, no multicast) into shared memory, for the
// regrouping engine's staged tile restore.  Addresses on 16-byte boundaries
// and sizes in multiples of 16 bytes (checked by the caller).

__device__ __forceinline__ unsigned
smem_addr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

/// An mbarrier with one expected arrival, visible to the bulk-copy unit.
__device__ __forceinline__ void
mbar_init(unsigned long long* mbar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

/// The one arrival of the mbarrier's current phase, which then completes
/// once `bytes` have been copied into shared memory.
__device__ __forceinline__ void
bulk_expect(unsigned long long* mbar, const unsigned bytes)
{
    unsigned long long state;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                 : "=l"(state)
                 : "r"(smem_addr(mbar)), "r"(bytes)
                 : "memory");
    (void)state;
}

/// One bulk copy of `bytes` from global to shared memory, counted on `mbar`.
__device__ __forceinline__ void
bulk_copy(void* dst, const void* src, const unsigned bytes, unsigned long long* mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(mbar))
                 : "memory");
}

/// Whether the mbarrier's phase of parity `phase` has completed.
__device__ __forceinline__ bool
mbar_try_wait(unsigned long long* mbar, const unsigned phase)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_addr(mbar)), "r"(phase)
                 : "memory");
    return ok != 0u;
}

/// Block-wide sum of three counters into global memory, one atomic per warp.
__device__ __forceinline__ void
flush_counters(unsigned long long* dst,
               unsigned long long a,
               unsigned long long b,
               unsigned long long c)
{
    for(int o = 16; o > 0; o >>= 1)
    {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if((threadIdx.x & 31) == 0)
    {
        if(a) atomicAdd(dst + 0, a);
        if(b) atomicAdd(dst + 1, b);
        if(c) atomicAdd(dst + 2, c);
    }
}
} // namespace loom_b200
