// Generated by loom_b200.codegen from loom_b200/ir/fib_u32.lir.
// Kernel IR digest b58369e636389a54; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_fib_u32 {

__constant__ unsigned kInstrTab[3] = {3, 4, 6};
__constant__ unsigned kLiveTab[3] = {4, 4, 16};

struct K
{
    static constexpr int kNumBlocks = 3;
    struct Regs
    {
        unsigned int r1; // n: u32
        unsigned int r2; // c: u32
        unsigned int r3; // cmp: u32
        unsigned int r4; // p: u32
        unsigned int r5; // i: u32
        unsigned int r6; // t: u32
    };

    __device__ __forceinline__ static void
    load_inputs(Regs& R, const Columns& c, const unsigned long long tid)
    {
        R.r1 = 0;
        R.r2 = 0;
        R.r3 = 0;
        R.r4 = 0;
        R.r5 = 0;
        R.r6 = 0;
        { // input n
            const unsigned int* col = static_cast<const unsigned int*>(c.p[0]);
            const unsigned int v = col ? col[tid] : static_cast<unsigned int>(tid);
            R.r1 = static_cast<unsigned int>(v);
        }
    }

    __device__ __forceinline__ static void
    store_outputs(const Regs& R, const Columns& c, const unsigned long long tid)
    {
        static_cast<unsigned int*>(c.p[1])[tid] = R.r2; // c
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
            R.r3 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r1) <= static_cast<unsigned int>(((unsigned int)0x1ull))));
            R.r2 = static_cast<unsigned int>(((R.r3) ? (R.r1) : (((unsigned int)0x1ull))));
            return ((R.r3) ? kHalt : 1);
        }
        case 1: // work
        {
            R.r4 = static_cast<unsigned int>(((unsigned int)0x0ull));
            R.r2 = static_cast<unsigned int>(((unsigned int)0x1ull));
            R.r5 = static_cast<unsigned int>(((unsigned int)0x2ull));
            return 2;
        }
        case 2: // loop
        {
            R.r6 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r4) + static_cast<unsigned int>(R.r2)));
            R.r4 = static_cast<unsigned int>(R.r2);
            R.r2 = static_cast<unsigned int>(R.r6);
            R.r5 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r5) + static_cast<unsigned int>(((unsigned int)0x1ull))));
            R.r3 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r5) <= static_cast<unsigned int>(R.r1)));
            return ((R.r3) ? 2 : kHalt);
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
        R.r3 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r1) <= static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r2 = static_cast<unsigned int>(((R.r3) ? (R.r1) : (((unsigned int)0x1ull))));
        if(R.r3) goto L_HALT; else goto L_B1;
    L_B1: // work
        if(++ctx.steps > ctx.max_steps) { ctx.flag(kStatusStepLimit); return; }
        if constexpr(kProf) count_block(ctx, 4u);
        R.r4 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r2 = static_cast<unsigned int>(((unsigned int)0x1ull));
        R.r5 = static_cast<unsigned int>(((unsigned int)0x2ull));
        goto L_B2;
    L_B2: // loop
        if(++ctx.steps > ctx.max_steps) { ctx.flag(kStatusStepLimit); return; }
        if constexpr(kProf) count_block(ctx, 6u);
        R.r6 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r4) + static_cast<unsigned int>(R.r2)));
        R.r4 = static_cast<unsigned int>(R.r2);
        R.r2 = static_cast<unsigned int>(R.r6);
        R.r5 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r5) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r3 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r5) <= static_cast<unsigned int>(R.r1)));
        if(R.r3) goto L_B2; else goto L_HALT;
    L_HALT:
        return;
    }

    __device__ __forceinline__ static void
    save(const int b, const Regs& R, const Columns& c, const unsigned slot)
    {
        switch(b)
        {
        case 0:
            static_cast<unsigned int*>(c.p[2])[slot] = R.r1;
            break;
        case 1:
            static_cast<unsigned int*>(c.p[2])[slot] = R.r1;
            break;
        case 2:
            static_cast<unsigned int*>(c.p[2])[slot] = R.r1;
            static_cast<unsigned int*>(c.p[3])[slot] = R.r2;
            static_cast<unsigned int*>(c.p[4])[slot] = R.r4;
            static_cast<unsigned int*>(c.p[5])[slot] = R.r5;
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
            R.r1 = static_cast<unsigned int*>(c.p[2])[slot];
            break;
        case 1:
            R.r1 = static_cast<unsigned int*>(c.p[2])[slot];
            break;
        case 2:
            R.r1 = static_cast<unsigned int*>(c.p[2])[slot];
            R.r2 = static_cast<unsigned int*>(c.p[3])[slot];
            R.r4 = static_cast<unsigned int*>(c.p[4])[slot];
            R.r5 = static_cast<unsigned int*>(c.p[5])[slot];
            break;
        default: break;
        }
    }

};

const int kInTypes[] = {LOOM_B200_U32};
const int kOutTypes[] = {LOOM_B200_U32};
const char* const kInNames[] = {"n"};
const char* const kOutNames[] = {"c"};
const int kStateTypes[] = {0, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const uint32_t kInstrs[] = {3, 4, 6};
const uint32_t kLive[] = {4, 4, 16};

const loom_b200_kernel_info kInfo = {
    "fib_u32", "b58369e636389a54", 1u, 1u, kInTypes, kOutTypes, kInNames, kOutNames,
    3u, 7u, 28u, 4u, kInstrs, kLive};

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

} } // namespace loom_b200::k_fib_u32

extern const loom_b200::KernelEntry loom_b200_entry_fib_u32;
const loom_b200::KernelEntry loom_b200_entry_fib_u32 = {
    &loom_b200::k_fib_u32::kInfo, 4, loom_b200::k_fib_u32::kStateTypes + 1,
    &loom_b200::k_fib_u32::launch_plain, &loom_b200::k_fib_u32::launch_regroup,
    &loom_b200::k_fib_u32::regroup_occupancy};
