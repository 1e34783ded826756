// Generated by loom_b200.codegen from loom_b200/ir/union_f32.lir.
// Kernel IR digest 3c99e81949745f96; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_union_f32 {

__constant__ unsigned kInstrTab[1] = {2};
__constant__ unsigned kLiveTab[1] = {4};

struct K
{
    static constexpr int kNumBlocks = 1;
    struct Regs
    {
        float r0; // i: f32
        unsigned int r1; // j: f32,u32
    };

    __device__ __forceinline__ static void
    load_inputs(Regs& R, const Columns& c, const unsigned long long tid)
    {
        R.r0 = 0;
        R.r1 = 0;
        { // input i
            const float* col = static_cast<const float*>(c.p[0]);
            const float v = col ? col[tid] : static_cast<float>(tid);
            R.r0 = static_cast<float>(v);
        }
    }

    __device__ __forceinline__ static void
    store_outputs(const Regs& R, const Columns& c, const unsigned long long tid)
    {
        static_cast<unsigned int*>(c.p[1])[tid] = R.r1; // j
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
            R.r1 = bitcast<unsigned int>(static_cast<float>(R.r0));
            R.r1 = static_cast<unsigned int>(bitcast<float>(R.r1));
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
        if constexpr(kProf) count_block(ctx, 2u);
        R.r1 = bitcast<unsigned int>(static_cast<float>(R.r0));
        R.r1 = static_cast<unsigned int>(bitcast<float>(R.r1));
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
            static_cast<float*>(c.p[2])[slot] = R.r0;
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
            R.r0 = static_cast<float*>(c.p[2])[slot];
            break;
        default: break;
        }
    }

};

const int kInTypes[] = {LOOM_B200_F32};
const int kOutTypes[] = {LOOM_B200_U32};
const char* const kInNames[] = {"i"};
const char* const kOutNames[] = {"j"};
const int kStateTypes[] = {0, LOOM_B200_F32};
const uint32_t kInstrs[] = {2};
const uint32_t kLive[] = {4};

const loom_b200_kernel_info kInfo = {
    "union_f32", "3c99e81949745f96", 1u, 1u, kInTypes, kOutTypes, kInNames, kOutNames,
    1u, 2u, 8u, 1u, kInstrs, kLive};

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

} } // namespace loom_b200::k_union_f32

extern const loom_b200::KernelEntry loom_b200_entry_union_f32;
const loom_b200::KernelEntry loom_b200_entry_union_f32 = {
    &loom_b200::k_union_f32::kInfo, 1, loom_b200::k_union_f32::kStateTypes + 1,
    &loom_b200::k_union_f32::launch_plain, &loom_b200::k_union_f32::launch_regroup,
    &loom_b200::k_union_f32::regroup_occupancy};
