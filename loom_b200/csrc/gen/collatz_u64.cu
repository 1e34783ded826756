// Generated by loom_b200.codegen from loom_b200/ir/collatz_u64.lir.
// Kernel IR digest 4d4fd74f333fab47; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_collatz_u64 {

__constant__ unsigned kInstrTab[2] = {3, 8};
__constant__ unsigned kLiveTab[2] = {8, 12};

struct K
{
    static constexpr int kNumBlocks = 2;
    struct Regs
    {
        unsigned long long r1; // n: u64
        unsigned int r2; // steps: u32
        unsigned long long r3; // cmp: u64
        unsigned long long r4; // odd: u64
        unsigned long long r5; // half: u64
        unsigned long long r6; // up: u64
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
            const unsigned long long* col = static_cast<const unsigned long long*>(c.p[0]);
            const unsigned long long v = col ? col[tid] : static_cast<unsigned long long>(tid);
            R.r1 = static_cast<unsigned long long>(v);
        }
    }

    __device__ __forceinline__ static void
    store_outputs(const Regs& R, const Columns& c, const unsigned long long tid)
    {
        static_cast<unsigned int*>(c.p[1])[tid] = R.r2; // steps
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
            R.r2 = static_cast<unsigned int>(((unsigned int)0x0ull));
            R.r3 = static_cast<unsigned long long>(static_cast<bool>(static_cast<unsigned long long>(R.r1) <= static_cast<unsigned long long>(((unsigned long long)0x1ull))));
            return ((R.r3) ? kHalt : 1);
        }
        case 1: // loop
        {
            R.r4 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) & static_cast<unsigned long long>(((unsigned long long)0x1ull))));
            R.r5 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) >> static_cast<unsigned long long>(((unsigned long long)0x1ull))));
            R.r6 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) * static_cast<unsigned long long>(((unsigned long long)0x3ull))));
            R.r6 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r6) + static_cast<unsigned long long>(((unsigned long long)0x1ull))));
            R.r1 = static_cast<unsigned long long>(((R.r4) ? (R.r6) : (R.r5)));
            R.r2 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r2) + static_cast<unsigned int>(((unsigned int)0x1ull))));
            R.r3 = static_cast<unsigned long long>(static_cast<bool>(static_cast<unsigned long long>(R.r1) != static_cast<unsigned long long>(((unsigned long long)0x1ull))));
            return ((R.r3) ? 1 : kHalt);
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
        R.r2 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r3 = static_cast<unsigned long long>(static_cast<bool>(static_cast<unsigned long long>(R.r1) <= static_cast<unsigned long long>(((unsigned long long)0x1ull))));
        if(R.r3) goto L_HALT; else goto L_B1;
    L_B1: // loop
        if(++ctx.steps > ctx.max_steps) { ctx.flag(kStatusStepLimit); return; }
        if constexpr(kProf) count_block(ctx, 8u);
        R.r4 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) & static_cast<unsigned long long>(((unsigned long long)0x1ull))));
        R.r5 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) >> static_cast<unsigned long long>(((unsigned long long)0x1ull))));
        R.r6 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r1) * static_cast<unsigned long long>(((unsigned long long)0x3ull))));
        R.r6 = static_cast<unsigned long long>(static_cast<unsigned long long>(static_cast<unsigned long long>(R.r6) + static_cast<unsigned long long>(((unsigned long long)0x1ull))));
        R.r1 = static_cast<unsigned long long>(((R.r4) ? (R.r6) : (R.r5)));
        R.r2 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r2) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r3 = static_cast<unsigned long long>(static_cast<bool>(static_cast<unsigned long long>(R.r1) != static_cast<unsigned long long>(((unsigned long long)0x1ull))));
        if(R.r3) goto L_B1; else goto L_HALT;
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
            static_cast<unsigned int*>(c.p[3])[slot] = R.r2;
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
            R.r2 = static_cast<unsigned int*>(c.p[3])[slot];
            break;
        default: break;
        }
    }

};

const int kInTypes[] = {LOOM_B200_U64};
const int kOutTypes[] = {LOOM_B200_U32};
const char* const kInNames[] = {"n"};
const char* const kOutNames[] = {"steps"};
const int kStateTypes[] = {0, LOOM_B200_U64, LOOM_B200_U32};
const uint32_t kInstrs[] = {3, 8};
const uint32_t kLive[] = {8, 12};

const loom_b200_kernel_info kInfo = {
    "collatz_u64", "4d4fd74f333fab47", 1u, 1u, kInTypes, kOutTypes, kInNames, kOutNames,
    2u, 7u, 52u, 2u, kInstrs, kLive};

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

} } // namespace loom_b200::k_collatz_u64

extern const loom_b200::KernelEntry loom_b200_entry_collatz_u64;
const loom_b200::KernelEntry loom_b200_entry_collatz_u64 = {
    &loom_b200::k_collatz_u64::kInfo, 2, loom_b200::k_collatz_u64::kStateTypes + 1,
    &loom_b200::k_collatz_u64::launch_plain, &loom_b200::k_collatz_u64::launch_regroup,
    &loom_b200::k_collatz_u64::regroup_occupancy};
