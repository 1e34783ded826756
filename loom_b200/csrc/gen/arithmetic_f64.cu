// Generated by loom_b200.codegen from loom_b200/ir/arithmetic_f64.lir.
// Kernel IR digest 69afbd9d697bba4a; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_arithmetic_f64 {

__constant__ unsigned kInstrTab[1] = {8};
__constant__ unsigned kLiveTab[1] = {24};

struct K
{
    static constexpr int kNumBlocks = 1;
    struct Regs
    {
        unsigned long long r0; // a: u64,f64
        double r1; // b: f64
        double r2; // c: f64
        double r3; // t: f64
    };

    __device__ __forceinline__ static void
    load_inputs(Regs& R, const Columns& c, const unsigned long long tid)
    {
        R.r0 = 0;
        R.r1 = 0;
        R.r2 = 0;
        R.r3 = 0;
        { // input a
            const double* col = static_cast<const double*>(c.p[0]);
            const double v = col ? col[tid] : static_cast<double>(tid);
            R.r0 = bitcast<unsigned long long>(static_cast<double>(v));
        }
        { // input b
            const double* col = static_cast<const double*>(c.p[1]);
            const double v = col ? col[tid] : static_cast<double>(tid);
            R.r1 = static_cast<double>(v);
        }
        { // input c
            const double* col = static_cast<const double*>(c.p[2]);
            const double v = col ? col[tid] : static_cast<double>(tid);
            R.r2 = static_cast<double>(v);
        }
    }

    __device__ __forceinline__ static void
    store_outputs(const Regs& R, const Columns& c, const unsigned long long tid)
    {
        static_cast<unsigned long long*>(c.p[3])[tid] = R.r0; // a
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
            R.r2 = static_cast<double>(static_cast<double>(-static_cast<double>(R.r2)));
            R.r3 = static_cast<double>(op_fma(bitcast<double>(R.r0), R.r1, R.r2));
            R.r0 = bitcast<unsigned long long>(static_cast<double>(static_cast<double>(static_cast<double>(bitcast<double>(R.r0)) * static_cast<double>(R.r1))));
            R.r0 = bitcast<unsigned long long>(static_cast<double>(static_cast<double>(static_cast<double>(bitcast<double>(R.r0)) + static_cast<double>(R.r2))));
            R.r0 = bitcast<unsigned long long>(static_cast<double>(static_cast<double>(static_cast<double>(R.r3) / static_cast<double>(bitcast<double>(R.r0)))));
            R.r0 = bitcast<unsigned long long>(static_cast<double>(static_cast<double>(static_cast<double>(bitcast<double>(R.r0)) - static_cast<double>((0x1.0000000000000p+0)))));
            R.r0 = bitcast<unsigned long long>(static_cast<double>(op_abs(static_cast<double>(bitcast<double>(R.r0)))));
            R.r0 = static_cast<unsigned long long>(static_cast<bool>(static_cast<double>(bitcast<double>(R.r0)) < static_cast<double>((0x1.0c6f7a0b5ed8dp-20))));
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
        if constexpr(kProf) count_block(ctx, 8u);
        R.r2 = static_cast<double>(static_cast<double>(-static_cast<double>(R.r2)));
        R.r3 = static_cast<double>(op_fma(bitcast<double>(R.r0), R.r1, R.r2));
        R.r0 = bitcast<unsigned long long>(static_cast<double>(static_cast<double>(static_cast<double>(bitcast<double>(R.r0)) * static_cast<double>(R.r1))));
        R.r0 = bitcast<unsigned long long>(static_cast<double>(static_cast<double>(static_cast<double>(bitcast<double>(R.r0)) + static_cast<double>(R.r2))));
        R.r0 = bitcast<unsigned long long>(static_cast<double>(static_cast<double>(static_cast<double>(R.r3) / static_cast<double>(bitcast<double>(R.r0)))));
        R.r0 = bitcast<unsigned long long>(static_cast<double>(static_cast<double>(static_cast<double>(bitcast<double>(R.r0)) - static_cast<double>((0x1.0000000000000p+0)))));
        R.r0 = bitcast<unsigned long long>(static_cast<double>(op_abs(static_cast<double>(bitcast<double>(R.r0)))));
        R.r0 = static_cast<unsigned long long>(static_cast<bool>(static_cast<double>(bitcast<double>(R.r0)) < static_cast<double>((0x1.0c6f7a0b5ed8dp-20))));
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
            static_cast<unsigned long long*>(c.p[4])[slot] = R.r0;
            static_cast<double*>(c.p[5])[slot] = R.r1;
            static_cast<double*>(c.p[6])[slot] = R.r2;
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
            R.r0 = static_cast<unsigned long long*>(c.p[4])[slot];
            R.r1 = static_cast<double*>(c.p[5])[slot];
            R.r2 = static_cast<double*>(c.p[6])[slot];
            break;
        default: break;
        }
    }

};

const int kInTypes[] = {LOOM_B200_F64, LOOM_B200_F64, LOOM_B200_F64};
const int kOutTypes[] = {LOOM_B200_U64};
const char* const kInNames[] = {"a", "b", "c"};
const char* const kOutNames[] = {"a"};
const int kStateTypes[] = {0, LOOM_B200_U64, LOOM_B200_F64, LOOM_B200_F64};
const uint32_t kInstrs[] = {8};
const uint32_t kLive[] = {24};

const loom_b200_kernel_info kInfo = {
    "arithmetic_f64", "69afbd9d697bba4a", 3u, 1u, kInTypes, kOutTypes, kInNames, kOutNames,
    1u, 4u, 32u, 3u, kInstrs, kLive};

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

} } // namespace loom_b200::k_arithmetic_f64

extern const loom_b200::KernelEntry loom_b200_entry_arithmetic_f64;
const loom_b200::KernelEntry loom_b200_entry_arithmetic_f64 = {
    &loom_b200::k_arithmetic_f64::kInfo, 3, loom_b200::k_arithmetic_f64::kStateTypes + 1,
    &loom_b200::k_arithmetic_f64::launch_plain, &loom_b200::k_arithmetic_f64::launch_regroup,
    &loom_b200::k_arithmetic_f64::regroup_occupancy};
