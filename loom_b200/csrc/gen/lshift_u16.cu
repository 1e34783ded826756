// Generated by loom_b200.codegen from loom_b200/ir/lshift_u16.lir.
// Kernel IR digest ae20da1d8bb81b44; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_lshift_u16 {

__constant__ unsigned kInstrTab[1] = {1};
__constant__ unsigned kLiveTab[1] = {4};

struct K
{
    static constexpr int kNumBlocks = 1;
    struct Regs
    {
        unsigned short r0; // a: u16
        unsigned short r1; // b: u16
    };

    __device__ __forceinline__ static void
    load_inputs(Regs& R, const Columns& c, const unsigned long long tid)
    {
        R.r0 = 0;
        R.r1 = 0;
        { // input a
            const unsigned short* col = static_cast<const unsigned short*>(c.p[0]);
            const unsigned short v = col ? col[tid] : static_cast<unsigned short>(tid);
            R.r0 = static_cast<unsigned short>(v);
        }
        { // input b
            const unsigned short* col = static_cast<const unsigned short*>(c.p[1]);
            const unsigned short v = col ? col[tid] : static_cast<unsigned short>(tid);
            R.r1 = static_cast<unsigned short>(v);
        }
    }

    __device__ __forceinline__ static void
    store_outputs(const Regs& R, const Columns& c, const unsigned long long tid)
    {
        static_cast<unsigned short*>(c.p[2])[tid] = R.r0; // a
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
            R.r0 = static_cast<unsigned short>(static_cast<unsigned short>(static_cast<unsigned short>(R.r0) << static_cast<unsigned short>(R.r1)));
            return kHalt;
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
        if constexpr(kProf) count_block(ctx, 1u);
        R.r0 = static_cast<unsigned short>(static_cast<unsigned short>(static_cast<unsigned short>(R.r0) << static_cast<unsigned short>(R.r1)));
        goto L_HALT;
    L_HALT:
        return;
    }

    __device__ __forceinline__ static void
    save(const int b, const Regs& R, const Columns& c, const unsigned slot)
    {
        switch(b)
        {
        case 0:
            static_cast<unsigned short*>(c.p[3])[slot] = R.r0;
            static_cast<unsigned short*>(c.p[4])[slot] = R.r1;
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
            R.r0 = static_cast<unsigned short*>(c.p[3])[slot];
            R.r1 = static_cast<unsigned short*>(c.p[4])[slot];
            break;
        default: break;
        }
    }

};

const int kInTypes[] = {LOOM_B200_U16, LOOM_B200_U16};
const int kOutTypes[] = {LOOM_B200_U16};
const char* const kInNames[] = {"a", "b"};
const char* const kOutNames[] = {"a"};
const int kStateTypes[] = {0, LOOM_B200_U16, LOOM_B200_U16};
const uint32_t kInstrs[] = {1};
const uint32_t kLive[] = {4};

const loom_b200_kernel_info kInfo = {
    "lshift_u16", "ae20da1d8bb81b44", 2u, 1u, kInTypes, kOutTypes, kInNames, kOutNames,
    1u, 2u, 4u, 2u, kInstrs, kLive};

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

} } // namespace loom_b200::k_lshift_u16

extern const loom_b200::KernelEntry loom_b200_entry_lshift_u16;
const loom_b200::KernelEntry loom_b200_entry_lshift_u16 = {
    &loom_b200::k_lshift_u16::kInfo, 2, loom_b200::k_lshift_u16::kStateTypes + 1,
    &loom_b200::k_lshift_u16::launch_plain, &loom_b200::k_lshift_u16::launch_regroup,
    &loom_b200::k_lshift_u16::regroup_occupancy};
