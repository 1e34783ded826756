// Generated by loom_b200.codegen from loom_b200/ir/fac_u64.lir.
// Kernel IR digest a649e9040b0c2ffa; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_fac_u64 {

__constant__ unsigned kInstrTab[3] = {3, 2, 4};
__constant__ unsigned kLiveTab[3] = {8, 8, 16};

struct K
{
    static constexpr int kNumBlocks = 3;
    struct Regs
    {
        unsigned long long r1; // a: u64
        unsigned long long r2; // cmp: u64
        unsigned long long r3; // c: u64
    };

    __device__ __forceinline__ static void
    load_inputs(Regs& R, const Columns& c, const unsigned long long tid)
    {
        R.r1 = 0;
        R.r2 = 0;
        R.r3 = 0;
        { // input a
            const unsigned long long* col = static_cast<const unsigned long long*>(c.p[0]);
            const unsigned long long v = col ? col[tid] : static_cast<unsigned long long>(tid);
            R.r1 = static_cast<unsigned long long>(v);
        }
    }

    __device__ __forceinline__ static void
    store_outputs(const Regs& R, const Columns& c, const unsigned long long tid)
    {
        static_cast<unsigned long long*>(c.p[1])[tid] = R.r1; // a
    }

    __device__ __forceinline__ static unsigned instr(const int b) { return kInstrTab[b]; }
    __device__ __forceinline__ static unsigned live_bytes(const int b) { return kLiveTab[b]; }

    __device__ __forceinline__ static int
    exec(const int b, Regs& R, Ctx& ctx)
    {
        (void)ctx;
        switch(b)
        {
        case 0: // START
        {
            R.r2 = static_cast<unsigned long long>(static_cast<bool>(static_cast<unsigned long long>(R.r1) <= static_cast<unsigned long long>(((unsigned long long)0x1ull))));
            R.r1 = static_cast<unsigned long long>(((R.r2) ? (((unsigned long long)0x1ull)) : (R.r1)));
            return ((R.r2) ? kHalt : 1);
        }
        case 1: // cinit
        {
            R.r3 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) - static_cast<unsigned long long>(((unsigned long long)0x1ull))));
            return 2;
        }
        case 2: // loop
        {
            R.r1 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) * static_cast<unsigned long long>(R.r3)));
            R.r3 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r3) - static_cast<unsigned long long>(((unsigned long long)0x1ull))));
            R.r2 = static_cast<unsigned long long>(static_cast<bool>(static_cast<unsigned long long>(R.r3) == static_cast<unsigned long long>(((unsigned long long)0x0ull))));
            return ((R.r2) ? kHalt : 2);
        }
        default: return kHalt;
        }
    }

    template <bool kProf>
    __device__ __forceinline__ static void
    run(Regs& R, Ctx& ctx)
    {
    L_B0: // START
        if(++ctx.steps > ctx.max_steps) { ctx.flag(kStatusStepLimit); return; }
        if constexpr(kProf) count_block(ctx, 3u);
        R.r2 = static_cast<unsigned long long>(static_cast<bool>(static_cast<unsigned long long>(R.r1) <= static_cast<unsigned long long>(((unsigned long long)0x1ull))));
        R.r1 = static_cast<unsigned long long>(((R.r2) ? (((unsigned long long)0x1ull)) : (R.r1)));
        if(R.r2) goto L_HALT; else goto L_B1;
    L_B1: // cinit
        if(++ctx.steps > ctx.max_steps) { ctx.flag(kStatusStepLimit); return; }
        if constexpr(kProf) count_block(ctx, 2u);
        R.r3 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) - static_cast<unsigned long long>(((unsigned long long)0x1ull))));
        goto L_B2;
    L_B2: // loop
        if(++ctx.steps > ctx.max_steps) { ctx.flag(kStatusStepLimit); return; }
        if constexpr(kProf) count_block(ctx, 4u);
        R.r1 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) * static_cast<unsigned long long>(R.r3)));
        R.r3 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r3) - static_cast<unsigned long long>(((unsigned long long)0x1ull))));
        R.r2 = static_cast<unsigned long long>(static_cast<bool>(static_cast<unsigned long long>(R.r3) == static_cast<unsigned long long>(((unsigned long long)0x0ull))));
        if(R.r2) goto L_HALT; else goto L_B2;
    L_HALT:
        return;
    }

    __device__ __forceinline__ static void
    save(const int b, const Regs& R, const Columns& c, const unsigned slot)
    {
        switch(b)
        {
        case 0:
            static_cast<unsigned long long*>(c.p[2])[slot] = R.r1;
            break;
        case 1:
            static_cast<unsigned long long*>(c.p[2])[slot] = R.r1;
            break;
        case 2:
            static_cast<unsigned long long*>(c.p[2])[slot] = R.r1;
            static_cast<unsigned long long*>(c.p[3])[slot] = R.r3;
            break;
        default: break;
        }
    }

    __device__ __forceinline__ static void
    restore(const int b, Regs& R, const Columns& c, const unsigned slot)
    {
        switch(b)
        {
        case 0:
            R.r1 = static_cast<unsigned long long*>(c.p[2])[slot];
            break;
        case 1:
            R.r1 = static_cast<unsigned long long*>(c.p[2])[slot];
            break;
        case 2:
            R.r1 = static_cast<unsigned long long*>(c.p[2])[slot];
            R.r3 = static_cast<unsigned long long*>(c.p[3])[slot];
            break;
        default: break;
        }
    }

};

const int kInTypes[] = {LOOM_B200_U64};
const int kOutTypes[] = {LOOM_B200_U64};
const char* const kInNames[] = {"a"};
const char* const kOutNames[] = {"a"};
const int kStateTypes[] = {0, LOOM_B200_U64, LOOM_B200_U64};
const uint32_t kInstrs[] = {3, 2, 4};
const uint32_t kLive[] = {8, 8, 16};

const loom_b200_kernel_info kInfo = {
    "fac_u64", "a649e9040b0c2ffa", 1u, 1u, kInTypes, kOutTypes, kInNames, kOutNames,
    3u, 4u, 32u, 2u, kInstrs, kLive};

cudaError_t launch_plain(const PlainLaunch& a)
{
    const unsigned long long grid = (a.n + a.block - 1) / a.block;
    if(grid == 0) return cudaSuccess;
    if(a.profile)
        plain_kernel<K, true><<<static_cast<unsigned>(grid), a.block, 0, a.stream>>>(
            a.cols, a.n, a.max_steps, a.status, a.counters);
    else
        plain_kernel<K, false><<<static_cast<unsigned>(grid), a.block, 0, a.stream>>>(
            a.cols, a.n, a.max_steps, a.status, a.counters);
    return cudaGetLastError();
}

cudaError_t launch_regroup(const RegroupLaunch& a)
{
    void* args[] = {const_cast<RegroupParams*>(&a.params)};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&regroup_kernel<K>),
                                       dim3(a.grid), dim3(a.block), args, 0, a.stream);
}

cudaError_t regroup_occupancy(int block, int* ctas)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, &regroup_kernel<K>, block, 0);
}

} } // namespace loom_b200::k_fac_u64

extern const loom_b200::KernelEntry loom_b200_entry_fac_u64;
const loom_b200::KernelEntry loom_b200_entry_fac_u64 = {
    &loom_b200::k_fac_u64::kInfo, 2, loom_b200::k_fac_u64::kStateTypes + 1,
    &loom_b200::k_fac_u64::launch_plain, &loom_b200::k_fac_u64::launch_regroup,
    &loom_b200::k_fac_u64::regroup_occupancy};
