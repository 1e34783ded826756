// Generated by loom_b200.codegen from loom_b200/ir/minmax_f64.lir.
// Kernel IR digest 7b49318e5ff56457; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_minmax_f64 {

__constant__ unsigned kInstrTab[1] = {3};
__constant__ unsigned kLiveTab[1] = {16};

struct K
{
    static constexpr int kNumBlocks = 1;
    struct Regs
    {
        double r0; // a: f64
        double r1; // b: f64
        unsigned long long r2; // r: u64
        double r3; // x: f64
        double r4; // n: f64
    };

    __device__ __forceinline__ static void
    load_inputs(Regs& R, const Columns& c, const unsigned long long tid)
    {
        R.r0 = 0;
        R.r1 = 0;
        R.r2 = 0;
        R.r3 = 0;
        R.r4 = 0;
        { // input a
            const double* col = static_cast<const double*>(c.p[0]);
            const double v = col ? col[tid] : static_cast<double>(tid);
            R.r0 = static_cast<double>(v);
        }
        { // input b
            const double* col = static_cast<const double*>(c.p[1]);
            const double v = col ? col[tid] : static_cast<double>(tid);
            R.r1 = static_cast<double>(v);
        }
    }

    __device__ __forceinline__ static void
    store_outputs(const Regs& R, const Columns& c, const unsigned long long tid)
    {
        static_cast<unsigned long long*>(c.p[2])[tid] = R.r2; // r
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
            R.r3 = static_cast<double>(op_max<double>(static_cast<double>(R.r0), static_cast<double>(R.r1)));
            R.r4 = static_cast<double>(op_min<double>(static_cast<double>(R.r0), static_cast<double>(R.r1)));
            R.r2 = static_cast<unsigned long long>(static_cast<bool>(static_cast<double>(R.r3) > static_cast<double>(R.r4)));
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
        if constexpr(kProf) count_block(ctx, 3u);
        R.r3 = static_cast<double>(op_max<double>(static_cast<double>(R.r0), static_cast<double>(R.r1)));
        R.r4 = static_cast<double>(op_min<double>(static_cast<double>(R.r0), static_cast<double>(R.r1)));
        R.r2 = static_cast<unsigned long long>(static_cast<bool>(static_cast<double>(R.r3) > static_cast<double>(R.r4)));
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
            static_cast<double*>(c.p[3])[slot] = R.r0;
            static_cast<double*>(c.p[4])[slot] = R.r1;
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
            R.r0 = static_cast<double*>(c.p[3])[slot];
            R.r1 = static_cast<double*>(c.p[4])[slot];
            break;
        default: break;
        }
    }

};

const int kInTypes[] = {LOOM_B200_F64, LOOM_B200_F64};
const int kOutTypes[] = {LOOM_B200_U64};
const char* const kInNames[] = {"a", "b"};
const char* const kOutNames[] = {"r"};
const int kStateTypes[] = {0, LOOM_B200_F64, LOOM_B200_F64};
const uint32_t kInstrs[] = {3};
const uint32_t kLive[] = {16};

const loom_b200_kernel_info kInfo = {
    "minmax_f64", "7b49318e5ff56457", 2u, 1u, kInTypes, kOutTypes, kInNames, kOutNames,
    1u, 5u, 40u, 2u, kInstrs, kLive};

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

} } // namespace loom_b200::k_minmax_f64

extern const loom_b200::KernelEntry loom_b200_entry_minmax_f64;
const loom_b200::KernelEntry loom_b200_entry_minmax_f64 = {
    &loom_b200::k_minmax_f64::kInfo, 2, loom_b200::k_minmax_f64::kStateTypes + 1,
    &loom_b200::k_minmax_f64::launch_plain, &loom_b200::k_minmax_f64::launch_regroup,
    &loom_b200::k_minmax_f64::regroup_occupancy};
