// Generated by loom_b200.codegen from loom_b200/ir/canonical_f32.lir.
// Kernel IR digest 36fb095f2df262b4; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_canonical_f32 {

__constant__ unsigned kInstrTab[1] = {3};
__constant__ unsigned kLiveTab[1] = {4};
__constant__ int kQueueBlock[1] = {0};
__constant__ unsigned kQuorumTab[1] = {7};
__constant__ unsigned kRankTab[1] = {0};

struct K
{
    static constexpr int kNumBlocks = 1;
    static constexpr int kNumQueues = 1;
    static constexpr int kRegroupMaxRegs = 64;
    static constexpr bool kSplitCallSites = true;
    struct Regs
    {
        unsigned int r0; // x: f32,u32
    };

    struct In
    {
        unsigned int v0; // x
    };

    // Reads the input columns of thread `tid` (a NULL column is iota).
    __device__ __forceinline__ static void
    load_in(In& in, const Columns& c, const unsigned long long tid)
    {
        in.v0 = load_input<unsigned int>(c, 0, tid);
        (void)in; (void)c; (void)tid;
    }

    // Loom's set_inputs: input variables written, every other register zero.
    // Only registers live at START (those its queue carries) are written:
    // the others are written before they are read on every path.
    __device__ __forceinline__ static void
    start(Regs& R, const In& in)
    {
        R.r0 = static_cast<unsigned int>(in.v0);
        (void)in;
    }

    __device__ __forceinline__ static void
    load_inputs(Regs& R, const Columns& c, const unsigned long long tid)
    {
        In in;
        load_in(in, c, tid);
        start(R, in);
    }

    __device__ __forceinline__ static void
    store_outputs(const Regs& R, const Columns& c, const unsigned long long tid)
    {
        static_cast<float*>(c.p[1])[col_index(c, tid)] = bitcast<float>(R.r0); // x
    }

    __device__ __forceinline__ static unsigned instr(const int b) { return kInstrTab[b]; }
    __device__ __forceinline__ static unsigned live_bytes(const int q) { return kLiveTab[q]; }
    __device__ __forceinline__ static int block_of(const int q) { return kQueueBlock[q]; }
    __device__ __forceinline__ static unsigned quorum(const int b) { return kQuorumTab[b]; }
    __device__ __forceinline__ static unsigned rank(const int b) { return kRankTab[b]; }
    static constexpr int kNumLong = 0;
    // j-th long block (most instructions first)
    __device__ __forceinline__ static int long_block(const int j)
    {
        (void)j;
        return -1;
    }

    static constexpr int kMaxQueuesPerBlock = 1;
    // j-th queue holding threads that stand at block b (-1: none).
    __device__ __forceinline__ static int
    queue_list(const int b, const int j)
    {
        return j == 0 ? b : -1;
    }

    // Queue a thread standing at block pc waits in: the block's own queue,
    // or for a dispatch block the queue of the context its register selects.
    __device__ __forceinline__ static int
    queue_of(const int pc, const Regs& R)
    {
        (void)R;
        return pc;
    }

    // Runs the lane's own path from block `entry` for at most `budget`
    // loop iterations (visits of a loop header); returns the block it
    // stopped at, or kHalt.  With `stop_heavy`, a block whose quorum is
    // above zero is entered only as the first block of the burst, when
    // the warp's vote chose it.  A block that loops on itself takes up
    // to `spin` further iterations without spending budget (a loop the
    // warp's lanes run together needs no step of its own per iteration).
    template <bool kProf>
    __device__ __forceinline__ static int
    run_burst(const int entry, Regs& R, Ctx& ctx, unsigned budget, const bool stop_heavy = false,
              unsigned spin = 0u)
    {
        (void)ctx;
        (void)stop_heavy;
        (void)spin;
        bool fresh = true; // no block run yet in this burst
        (void)fresh;
        switch(entry)
        {
        case 0: goto L_B0;
        default: return kHalt;
        }
    L_B0: // START
        if(stop_heavy && !fresh) return 0;
    L_B0_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 0, 3u);
        R.r0 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r0) >> static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r0 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r0) | static_cast<unsigned int>(((unsigned int)0x3f800000ull))));
        R.r0 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r0)) - static_cast<float>((0x1.0000000000000p+0f)))));
        goto L_HALT;
    L_HALT:
        return kHalt;
    }

    static constexpr unsigned long long kRowBytes = 8ull;
    __device__ __forceinline__ static void
    save(const int q, const Regs& R, char* st, const unsigned cap, const unsigned par,
         const unsigned idx, const unsigned tid)
    {
        char* base = st + static_cast<unsigned long long>(par) * kRowBytes * cap;
        switch(q)
        {
        case 0: // START
        {
            {
                uint2 v0;
                v0.x = bitcast<unsigned>(R.r0);
                v0.y = tid;
                reinterpret_cast<uint2*>(base + 0ull * cap)[idx] = v0;
            }
            return;
        }
        default: return;
        }
    }

    __device__ __forceinline__ static unsigned
    restore(const int q, Regs& R, const char* st, const unsigned cap, const unsigned par,
            const unsigned idx)
    {
        const char* base = st + static_cast<unsigned long long>(par) * kRowBytes * cap;
        switch(q)
        {
        case 0: // START
        {
            const uint2 v0 = reinterpret_cast<const uint2*>(base + 0ull * cap)[idx];
            R.r0 = bitcast<unsigned int>(v0.x);
            return v0.y;
        }
        default: return 0xffffffffu;
        }
    }

    // bytes of one queue entry's slots, the largest over the queues
    static constexpr unsigned kMaxStageRow = 16u;
    // Lane 0 of a warp: copies the full tile [toff, toff + 32) of queue q
    // (state half `base`) into `stage` (32 x kMaxStageRow bytes of shared
    // memory) with one bulk copy per slot column, completing on the
    // mbarrier at `mbar`; false (nothing issued) when an address is not on
    // a 16-byte boundary.
    __device__ __forceinline__ static bool
    bulk_issue(const int q, unsigned char* stage, const char* base, const unsigned cap, const unsigned toff,
               unsigned long long* mbar)
    {
        unsigned bytes = 0;
        switch(q)
        {
        case 0: bytes = 256u; break;
        default: return false;
        }
        if((reinterpret_cast<unsigned long long>(base) | reinterpret_cast<unsigned long long>(stage)) & 15ull) return false;
        bulk_expect(mbar, bytes);
        switch(q)
        {
        case 0:
            bulk_copy(stage + 0u, base + 0ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        default: break;
        }
        return true;
    }

    // A lane's entry of a tile staged by bulk_issue; returns its thread id.
    __device__ __forceinline__ static unsigned
    restore_stage(const int q, Regs& R, const unsigned char* stage, const unsigned lane)
    {
        switch(q)
        {
        case 0:
        {
            const uint2 v0 = reinterpret_cast<const uint2*>(stage + 0u)[lane];
            R.r0 = bitcast<unsigned int>(v0.x);
            return v0.y;
        }
        default: return 0xffffffffu;
        }
    }
};

const int kInTypes[] = {LOOM_B200_U32};
const int kOutTypes[] = {LOOM_B200_F32};
const char* const kInNames[] = {"x"};
const char* const kOutNames[] = {"x"};
const uint32_t kInstrs[] = {3};
const uint32_t kLive[] = {4};

const loom_b200_kernel_info kInfo = {
    "canonical_f32", "36fb095f2df262b4", 1u, 1u, kInTypes, kOutTypes, kInNames, kOutNames,
    1u, 1u, 4u, 1u, kInstrs, kLive};

const uint32_t kQRegs0[] = {0u};
const int kQTypes0[] = {LOOM_B200_U32};
const char* const kQNames0[] = {"x"};
const unsigned long long kQOffs0[] = {0ull};
const unsigned kQSubs0[] = {0u};
const unsigned kQWidths0[] = {8u};
const loom_b200_queue_layout kQueues[] = {
    {0u, -1, 1u, kQRegs0, kQTypes0, kQNames0},
};
const QueueSegment kSegments[] = {
    {kQOffs0, kQSubs0, kQWidths0, 0ull, 4u, 8u},
};

cudaError_t launch_plain(const PlainLaunch& a)
{
    const unsigned long long grid = (a.n + a.block - 1) / a.block;
    if(grid == 0) return cudaSuccess;
    if(a.profile)
        plain_kernel<K, true><<<static_cast<unsigned>(grid), a.block, 0, a.stream>>>(
            a.cols, a.first, a.n, a.max_steps, a.status, a.counters);
    else
        plain_kernel<K, false><<<static_cast<unsigned>(grid), a.block, 0, a.stream>>>(
            a.cols, a.first, a.n, a.max_steps, a.status, a.counters);
    return cudaGetLastError();
}

const unsigned kRegCaps[] = {64u, 40u, 48u};

/// The megakernel at register cap `regs` (0: the default), in its form
/// for launches that never park when `park` is false; profiled launches
/// and launches with the staged restore (`bulk`) use the default cap and
/// the parking form.  NULL: no such cap compiled.
const void* regroup_fn(unsigned regs, bool profile, bool bulk, bool park)
{
    if(profile) return reinterpret_cast<const void*>(&regroup_kernel<K, true, K::kRegroupMaxRegs, true>);
    if(bulk) return reinterpret_cast<const void*>(&regroup_kernel<K, false, K::kRegroupMaxRegs, true>);
    switch(regs)
    {
    case 0u:
    case 64u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 64, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 64, false, false>);
    case 40u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 40, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 40, false, false>);
    case 48u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 48, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 48, false, false>);
    default: return nullptr;
    }
}

cudaError_t launch_regroup(const RegroupLaunch& a)
{
    void* args[] = {const_cast<RegroupParams*>(&a.params)};
    const void* fn = regroup_fn(a.regs, a.profile, a.params.bulk_restore != 0u, a.park);
    if(!fn) return cudaErrorInvalidValue;
    if(a.dyn_smem)
    {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(a.dyn_smem));
        if(e != cudaSuccess) return e;
    }
    if(a.ordinary && a.params.slice_rounds == 1u)
        return cudaLaunchKernel(fn, dim3(a.grid), dim3(a.block), args, a.dyn_smem, a.stream);
    return cudaLaunchCooperativeKernel(fn, dim3(a.grid), dim3(a.block), args, a.dyn_smem, a.stream);
}

cudaError_t regroup_occupancy(int block, bool profile, unsigned regs, unsigned dyn_smem, bool park, int* ctas)
{
    const void* fn = regroup_fn(regs, profile, dyn_smem != 0u, park);
    if(!fn) return cudaErrorInvalidValue;
    if(dyn_smem)
    {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(dyn_smem));
        if(e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, dyn_smem);
}

} } // namespace loom_b200::k_canonical_f32

extern const loom_b200::KernelEntry loom_b200_entry_canonical_f32;
const loom_b200::KernelEntry loom_b200_entry_canonical_f32 = {
    &loom_b200::k_canonical_f32::kInfo, loom_b200::k_canonical_f32::K::kRowBytes, 1,
    &loom_b200::k_canonical_f32::launch_plain, &loom_b200::k_canonical_f32::launch_regroup,
    &loom_b200::k_canonical_f32::regroup_occupancy,
    loom_b200::k_canonical_f32::kQueues, loom_b200::k_canonical_f32::kSegments,
    loom_b200::k_canonical_f32::kRegCaps, 3u, loom_b200::k_canonical_f32::K::kMaxStageRow};
