// Generated by loom_b200.codegen from loom_b200/ir/primary_const_b20_256.lir.
// Kernel IR digest 1f441c05ae8a8bdc; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_primary_const_b20_256 {

__constant__ unsigned kInstrTab[33] = {25, 335, 31, 11, 20, 3, 19, 10, 13, 22, 7, 28, 12, 15, 7, 7, 25, 3, 3, 3, 5, 11, 4, 3, 2, 4, 13, 15, 14, 16, 13, 20, 4};
__constant__ unsigned kLiveTab[33] = {8, 48, 84, 148, 140, 140, 132, 160, 148, 120, 88, 80, 132, 124, 108, 88, 80, 100, 96, 96, 100, 100, 96, 92, 92, 88, 80, 92, 108, 100, 88, 52, 20};
__constant__ int kQueueBlock[33] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32};
__constant__ unsigned kQuorumTab[33] = {26, 28, 6, 0, 0, 0, 0, 0, 0, 0, 0, 5, 0, 0, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 6, 0};
__constant__ unsigned kRankTab[33] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 22, 23, 18, 19, 20, 21, 24, 25, 26, 27, 28, 29, 30, 31, 32};

struct K
{
    static constexpr int kNumBlocks = 33;
    static constexpr int kNumQueues = 33;
    static constexpr int kRegroupMaxRegs = 64;
    static constexpr bool kSplitCallSites = false;
    struct Regs
    {
        unsigned int r1; // ppp: u32
        float r2; // L0: f32
        float r3; // L1: f32
        float r4; // L2: f32
        unsigned int r5; // rc: u32
        unsigned int r6; // d0: f32,u32
        unsigned int r7; // d1: f32,u32
        unsigned int r8; // c0: u32
        unsigned int r9; // c1: u32
        unsigned int r10; // tmp1: u32,f32
        unsigned int r11; // tmp2: u32,f32
        float r12; // pp0: f32
        float r13; // pp1: f32
        unsigned int r14; // tmp0: u32,f32
        float r15; // pw: f32
        unsigned int r16; // rpt: u32
        unsigned int r17; // sc: u32
        unsigned int r18; // u0: f32,u32
        unsigned int r19; // u1: f32,u32
        float r20; // o0: f32
        float r21; // o1: f32
        float r22; // o2: f32
        float r23; // clr0: f32
        float r24; // clr1: f32
        float r25; // clr2: f32
        unsigned int r26; // depth: u32
        float r27; // d2: f32
        float r28; // vr00: f32
        float r29; // vr01: f32
        float r30; // vr02: f32
        float r31; // t: f32
        unsigned int r32; // pid: u32
        unsigned int r33; // rp: u32
        float r34; // vr10: f32
        unsigned int r35; // vr11: u32,f32
        float r36; // vr12: f32
        float r37; // vr20: f32
        float r38; // vr21: f32
        float r39; // vr22: f32
        float r40; // vr30: f32
        float r41; // vr31: f32
        float r42; // vr32: f32
        float r43; // vr40: f32
        float r44; // vr41: f32
        float r45; // vr42: f32
        float r46; // vr50: f32
        float r47; // vr51: f32
        float r48; // vr52: f32
        unsigned int r49; // hit: u32,f32
        float r50; // vr60: f32
        float r51; // vr61: f32
        float r52; // vr62: f32
        unsigned int r53; // ct: u32,f32
    };

    struct In
    {
        unsigned int v0; // ppp
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
        R.r53 = 0;
        R.r1 = static_cast<unsigned int>(in.v0);
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
        static_cast<float*>(c.p[1])[col_index(c, tid)] = R.r2; // L0
        static_cast<float*>(c.p[2])[col_index(c, tid)] = R.r3; // L1
        static_cast<float*>(c.p[3])[col_index(c, tid)] = R.r4; // L2
        static_cast<unsigned int*>(c.p[4])[col_index(c, tid)] = R.r5; // rc
        static_cast<unsigned int*>(c.p[5])[col_index(c, tid)] = R.r1; // ppp
    }

    __device__ __forceinline__ static unsigned instr(const int b) { return kInstrTab[b]; }
    __device__ __forceinline__ static unsigned live_bytes(const int q) { return kLiveTab[q]; }
    __device__ __forceinline__ static int block_of(const int q) { return kQueueBlock[q]; }
    __device__ __forceinline__ static unsigned quorum(const int b) { return kQuorumTab[b]; }
    __device__ __forceinline__ static unsigned rank(const int b) { return kRankTab[b]; }
    static constexpr int kNumLong = 1;
    // j-th long block (most instructions first)
    __device__ __forceinline__ static int long_block(const int j)
    {
        switch(j)
        {
        case 0: return 1;
        default: return -1;
        }
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
        case 1: goto L_B1;
        case 2: goto L_B2;
        case 3: goto L_B3;
        case 4: goto L_B4;
        case 5: goto L_B5;
        case 6: goto L_B6;
        case 7: goto L_B7;
        case 8: goto L_B8;
        case 9: goto L_B9;
        case 10: goto L_B10;
        case 11: goto L_B11;
        case 12: goto L_B12;
        case 13: goto L_B13;
        case 14: goto L_B14;
        case 15: goto L_B15;
        case 16: goto L_B16;
        case 17: goto L_B17;
        case 18: goto L_B18;
        case 19: goto L_B19;
        case 20: goto L_B20;
        case 21: goto L_B21;
        case 22: goto L_B22;
        case 23: goto L_B23;
        case 24: goto L_B24;
        case 25: goto L_B25;
        case 26: goto L_B26;
        case 27: goto L_B27;
        case 28: goto L_B28;
        case 29: goto L_B29;
        case 30: goto L_B30;
        case 31: goto L_B31;
        case 32: goto L_B32;
        default: return kHalt;
        }
    L_B0: // START
        if(stop_heavy && !fresh) return 0;
    L_B0_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 0, 25u);
        R.r6 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r1) >> static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r7 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r1) & static_cast<unsigned int>(((unsigned int)0xffffull))));
        R.r8 = static_cast<unsigned int>(R.r6);
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) * static_cast<unsigned int>(((unsigned int)0x100ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) + static_cast<unsigned int>(R.r7)));
        R.r9 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p+8f)));
        R.r11 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p+8f)));
        R.r12 = static_cast<float>(R.r6);
        R.r13 = static_cast<float>(R.r7);
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) / static_cast<float>(bitcast<float>(R.r11)))));
        R.r15 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) / static_cast<float>(bitcast<float>(R.r10))));
        R.r15 = static_cast<float>(static_cast<float>(static_cast<float>(R.r15) * static_cast<float>((0x1.4000000000000p+4f))));
        R.r12 = static_cast<float>(static_cast<float>(static_cast<float>(R.r12) / static_cast<float>(bitcast<float>(R.r10))));
        R.r12 = static_cast<float>(static_cast<float>(static_cast<float>(R.r12) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r12 = static_cast<float>(static_cast<float>(static_cast<float>(R.r12) * static_cast<float>(bitcast<float>(R.r14))));
        R.r13 = static_cast<float>(static_cast<float>(static_cast<float>(R.r13) / static_cast<float>(bitcast<float>(R.r11))));
        R.r13 = static_cast<float>(static_cast<float>(static_cast<float>(R.r13) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r2 = static_cast<float>((0x0.0p+0f));
        R.r3 = static_cast<float>((0x0.0p+0f));
        R.r4 = static_cast<float>((0x0.0p+0f));
        R.r5 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r16 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r17 = static_cast<unsigned int>(((unsigned int)0x0ull));
        goto L_B1;
    L_B1: // roll
        if(stop_heavy && !fresh) return 1;
    L_B1_again:
        if(budget == 0u) return 1;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 1, 335u);
        R.r18 = static_cast<unsigned int>(R.r8);
        R.r19 = static_cast<unsigned int>(R.r9);
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x3ull))));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x7ull))));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(R.r19)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r18)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) + static_cast<unsigned int>(((unsigned int)0x54dull))));
        R.r10 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r14) < static_cast<unsigned int>(R.r8)));
        R.r11 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r9) + static_cast<unsigned int>(R.r14)));
        R.r9 = static_cast<unsigned int>(((R.r10) ? (R.r11) : (R.r9)));
        R.r8 = static_cast<unsigned int>(((R.r10) ? (((unsigned int)0x0ull)) : (R.r14)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) >> static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) | static_cast<unsigned int>(((unsigned int)0x3f800000ull))));
        R.r18 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r18)) - static_cast<float>((0x1.0000000000000p+0f)))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >> static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) | static_cast<unsigned int>(((unsigned int)0x3f800000ull))));
        R.r19 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r19)) - static_cast<float>((0x1.0000000000000p+0f)))));
        R.r20 = static_cast<float>((0x0.0p+0f));
        R.r21 = static_cast<float>((0x0.0p+0f));
        R.r22 = static_cast<float>((0x1.0000000000000p+1f));
        R.r6 = bitcast<unsigned int>(static_cast<float>(R.r12));
        R.r7 = bitcast<unsigned int>(static_cast<float>(R.r13));
        R.r23 = static_cast<float>((0x0.0p+0f));
        R.r24 = static_cast<float>((0x0.0p+0f));
        R.r25 = static_cast<float>((0x0.0p+0f));
        R.r26 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r17 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r17) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r15) * static_cast<float>((0x1.0000000000000p-1f)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) - static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) - static_cast<float>(bitcast<float>(R.r14)))));
        R.r18 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r18)) * static_cast<float>(R.r15))));
        R.r19 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r19)) * static_cast<float>(R.r15))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) + static_cast<float>(bitcast<float>(R.r18)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) + static_cast<float>(bitcast<float>(R.r19)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>((0x1.6d9b200000000p+0f)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>((0x1.6d9b200000000p+0f)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r6)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r7)))));
        R.r27 = static_cast<float>((-0x1.0000000000000p+0f));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r27, R.r27, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r27 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(bitcast<float>(R.r14))));
        R.r28 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>((0x1.0624de0000000p-10f))));
        R.r29 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>((0x1.0624de0000000p-10f))));
        R.r30 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>((0x1.0624de0000000p-10f))));
        R.r20 = static_cast<float>(static_cast<float>(static_cast<float>(R.r20) + static_cast<float>(R.r28)));
        R.r21 = static_cast<float>(static_cast<float>(static_cast<float>(R.r21) + static_cast<float>(R.r29)));
        R.r22 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) + static_cast<float>(R.r30)));
        R.r31 = static_cast<float>((0x1.e848000000000p+19f));
        R.r32 = static_cast<unsigned int>(((unsigned int)0xcull));
        R.r33 = static_cast<unsigned int>(((unsigned int)0x0ull));
        goto L_B2;
    L_B2: // traverse_box
        if(stop_heavy && !fresh) return 2;
    L_B2_again:
        if(budget == 0u) return 2;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 2, 31u);
        R.r28 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : ((R.r33) == 2 ? (0x1.0000000000000p+0f) : ((R.r33) == 3 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r29 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : ((R.r33) == 2 ? (-0x1.0000000000000p+0f) : ((R.r33) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r30 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (0x1.0000000000000p+0f) : ((R.r33) == 1 ? (0x1.0000000000000p+0f) : ((R.r33) == 2 ? (-0x1.0000000000000p+0f) : ((R.r33) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r34 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : ((R.r33) == 2 ? (0x1.0000000000000p+0f) : ((R.r33) == 3 ? (-0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r35 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : ((R.r33) == 2 ? (-0x1.0000000000000p+0f) : ((R.r33) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f))))))));
        R.r36 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : ((R.r33) == 2 ? (0x1.0000000000000p+0f) : ((R.r33) == 3 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r37 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : ((R.r33) == 2 ? (0x1.0000000000000p+0f) : ((R.r33) == 3 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r38 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (0x1.0000000000000p+0f) : ((R.r33) == 2 ? (0x1.0000000000000p+0f) : ((R.r33) == 3 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r39 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : ((R.r33) == 2 ? (0x1.0000000000000p+0f) : ((R.r33) == 3 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r40 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : ((R.r33) == 2 ? (0x1.0000000000000p+0f) : ((R.r33) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r41 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (0x1.0000000000000p+0f) : ((R.r33) == 2 ? (0x1.0000000000000p+0f) : ((R.r33) == 3 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r42 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (0x1.0000000000000p+0f) : ((R.r33) == 2 ? (-0x1.0000000000000p+0f) : ((R.r33) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r40) - static_cast<float>(R.r28)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r41) - static_cast<float>(R.r29)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r30)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r34) - static_cast<float>(R.r28)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r35)) - static_cast<float>(R.r29)));
        R.r48 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) - static_cast<float>(R.r30)));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r47))));
        R.r50 = static_cast<float>(op_fma(bitcast<float>(R.r7), R.r48, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r48))));
        R.r51 = static_cast<float>(op_fma(R.r27, R.r46, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r46))));
        R.r52 = static_cast<float>(op_fma(bitcast<float>(R.r6), R.r47, (-(bitcast<float>(R.r49)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r43, R.r50, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r44, R.r51, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r52, bitcast<float>(R.r14))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r14)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r10)) >= static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r49) goto L_B3; else goto L_B10;
    L_B3: // isect_quad_l1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 3, 11u);
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r20) - static_cast<float>(R.r28)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r21) - static_cast<float>(R.r29)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r30)));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r43, R.r50, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r44, R.r51, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r52, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r10)) >= static_cast<float>((0x0.0p+0f))));
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r10)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r49) goto L_B4; else goto L_B10;
    L_B4: // isect_quad_l2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 4, 20u);
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r40) - static_cast<float>(R.r28)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r41) - static_cast<float>(R.r29)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r30)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r20) - static_cast<float>(R.r28)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r21) - static_cast<float>(R.r29)));
        R.r48 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r30)));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r48) * static_cast<float>(R.r44))));
        R.r50 = static_cast<float>(op_fma(R.r47, R.r45, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>(R.r45))));
        R.r51 = static_cast<float>(op_fma(R.r48, R.r43, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r47) * static_cast<float>(R.r43))));
        R.r52 = static_cast<float>(op_fma(R.r46, R.r44, (-(bitcast<float>(R.r49)))));
        R.r11 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r11 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r50, bitcast<float>(R.r11))));
        R.r11 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r51, bitcast<float>(R.r11))));
        R.r11 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r27, R.r52, bitcast<float>(R.r11))));
        R.r11 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r11)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r11)) >= static_cast<float>((0x0.0p+0f))));
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r11)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r49) goto L_B5; else goto L_B10;
    L_B5: // isect_quad_l3
        fresh = false;
        if constexpr(kProf) count_block(ctx, 5, 3u);
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) + static_cast<float>(bitcast<float>(R.r11)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r53)) > static_cast<float>((0x1.0000000000000p+0f))));
        if(R.r49) goto L_B6; else goto L_B9;
    L_B6: // isect_quad_l4
        fresh = false;
        if constexpr(kProf) count_block(ctx, 6, 19u);
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r34) - static_cast<float>(R.r37)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r35)) - static_cast<float>(R.r38)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) - static_cast<float>(R.r39)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r40) - static_cast<float>(R.r37)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r41) - static_cast<float>(R.r38)));
        R.r48 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r39)));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r47))));
        R.r50 = static_cast<float>(op_fma(bitcast<float>(R.r7), R.r48, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r48))));
        R.r51 = static_cast<float>(op_fma(R.r27, R.r46, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r46))));
        R.r52 = static_cast<float>(op_fma(bitcast<float>(R.r6), R.r47, (-(bitcast<float>(R.r49)))));
        R.r53 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r43, R.r50, bitcast<float>(R.r53))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r44, R.r51, bitcast<float>(R.r53))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r52, bitcast<float>(R.r53))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r53)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r49)) >= static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r49) goto L_B7; else goto L_B10;
    L_B7: // isect_quad_l5
        fresh = false;
        if constexpr(kProf) count_block(ctx, 7, 10u);
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r20) - static_cast<float>(R.r37)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r21) - static_cast<float>(R.r38)));
        R.r48 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r39)));
        R.r49 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, R.r50, bitcast<float>(R.r49))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, R.r51, bitcast<float>(R.r49))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r48, R.r52, bitcast<float>(R.r49))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) / static_cast<float>(bitcast<float>(R.r53)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r49)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r49) goto L_B8; else goto L_B10;
    L_B8: // isect_quad_l6
        fresh = false;
        if constexpr(kProf) count_block(ctx, 8, 13u);
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r48) * static_cast<float>(R.r44))));
        R.r50 = static_cast<float>(op_fma(R.r47, R.r45, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>(R.r45))));
        R.r51 = static_cast<float>(op_fma(R.r48, R.r43, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r47) * static_cast<float>(R.r43))));
        R.r52 = static_cast<float>(op_fma(R.r46, R.r44, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r50, bitcast<float>(R.r49))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r51, bitcast<float>(R.r49))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r27, R.r52, bitcast<float>(R.r49))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) / static_cast<float>(bitcast<float>(R.r53)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r49)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r49) goto L_B9; else goto L_B10;
    L_B9: // isect_quad_l7
        fresh = false;
        if constexpr(kProf) count_block(ctx, 9, 22u);
        R.r40 = static_cast<float>(static_cast<float>(static_cast<float>(R.r40) - static_cast<float>(R.r28)));
        R.r41 = static_cast<float>(static_cast<float>(static_cast<float>(R.r41) - static_cast<float>(R.r29)));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r30)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r20) - static_cast<float>(R.r28)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r21) - static_cast<float>(R.r29)));
        R.r48 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r30)));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r48) * static_cast<float>(R.r41))));
        R.r50 = static_cast<float>(op_fma(R.r47, R.r42, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>(R.r42))));
        R.r51 = static_cast<float>(op_fma(R.r48, R.r40, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r47) * static_cast<float>(R.r40))));
        R.r52 = static_cast<float>(op_fma(R.r46, R.r41, (-(bitcast<float>(R.r49)))));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(R.r34) - static_cast<float>(R.r28)));
        R.r35 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r35)) - static_cast<float>(R.r29))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) - static_cast<float>(R.r30)));
        R.r53 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r34, R.r50, bitcast<float>(R.r53))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r35), R.r51, bitcast<float>(R.r53))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r36, R.r52, bitcast<float>(R.r53))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r53)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r53)) >= static_cast<float>((0x0.0p+0f))));
        goto L_B10;
    L_B10: // isect_quad_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 10, 7u);
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r53)) < static_cast<float>(R.r31))));
        R.r31 = static_cast<float>(((R.r49) ? (bitcast<float>(R.r53)) : (R.r31)));
        R.r32 = static_cast<unsigned int>(((R.r49) ? (R.r33) : (R.r32)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r33) == static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r33 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r33) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r33 = static_cast<unsigned int>(((R.r14) ? (((unsigned int)0x0ull)) : (R.r33)));
        if(R.r14) goto L_B11; else goto L_B2;
    L_B11: // traverse_tetrahedron
        if(stop_heavy && !fresh) return 11;
    L_B11_again:
        if(budget == 0u) return 11;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 11, 28u);
        R.r28 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.935f360000000p-1f) : ((R.r33) == 1 ? (-0x1.157b7e0000000p-1f) : (0x1.09d1420000000p-3f)))));
        R.r29 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))));
        R.r30 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.2cf8d20000000p-1f) : ((R.r33) == 1 ? (0x1.51b56e0000000p-2f) : (-0x1.5e2a2e0000000p-2f)))));
        R.r34 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.157b7e0000000p-1f) : ((R.r33) == 1 ? (0x1.09d1420000000p-3f) : (-0x1.935f360000000p-1f)))));
        R.r35 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r33) == 0 ? (-0x1.0000000000000p+0f) : ((R.r33) == 1 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f))))));
        R.r36 = static_cast<float>(static_cast<float>(((R.r33) == 0 ? (0x1.51b56e0000000p-2f) : ((R.r33) == 1 ? (-0x1.5e2a2e0000000p-2f) : (-0x1.2cf8d20000000p-1f)))));
        R.r37 = static_cast<float>((-0x1.9999980000000p-2f));
        R.r38 = static_cast<float>((-0x1.6b0f960000000p-3f));
        R.r39 = static_cast<float>((-0x1.9999980000000p-3f));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(R.r34) - static_cast<float>(R.r28)));
        R.r35 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r35)) - static_cast<float>(R.r29))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) - static_cast<float>(R.r30)));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) - static_cast<float>(R.r28)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) - static_cast<float>(R.r29)));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r39) - static_cast<float>(R.r30)));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r38))));
        R.r40 = static_cast<float>(op_fma(bitcast<float>(R.r7), R.r39, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r39))));
        R.r41 = static_cast<float>(op_fma(R.r27, R.r37, (-(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r37))));
        R.r42 = static_cast<float>(op_fma(bitcast<float>(R.r6), R.r38, (-(bitcast<float>(R.r49)))));
        R.r53 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r34, R.r40, bitcast<float>(R.r53))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r35), R.r41, bitcast<float>(R.r53))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r36, R.r42, bitcast<float>(R.r53))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r53)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r49) goto L_B12; else goto L_B15;
    L_B12: // isect_triangle_mid1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 12, 12u);
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(bitcast<float>(R.r53)))));
        R.r28 = static_cast<float>(static_cast<float>(static_cast<float>(R.r20) - static_cast<float>(R.r28)));
        R.r29 = static_cast<float>(static_cast<float>(static_cast<float>(R.r21) - static_cast<float>(R.r29)));
        R.r30 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r30)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r28, R.r40, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r29, R.r41, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r30, R.r42, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r53)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x0.0p+0f))));
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r49) goto L_B13; else goto L_B15;
    L_B13: // isect_triangle_mid2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 13, 15u);
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r30) * static_cast<float>(bitcast<float>(R.r35)))));
        R.r40 = static_cast<float>(op_fma(R.r29, R.r36, (-(bitcast<float>(R.r10)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r28) * static_cast<float>(R.r36))));
        R.r41 = static_cast<float>(op_fma(R.r30, R.r34, (-(bitcast<float>(R.r10)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r29) * static_cast<float>(R.r34))));
        R.r42 = static_cast<float>(op_fma(R.r28, bitcast<float>(R.r35), (-(bitcast<float>(R.r10)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r40, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r41, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r27, R.r42, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) * static_cast<float>(bitcast<float>(R.r53)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r10)) >= static_cast<float>((0x0.0p+0f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) + static_cast<float>(bitcast<float>(R.r10)))));
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r49) goto L_B14; else goto L_B15;
    L_B14: // isect_triangle_mid3
        fresh = false;
        if constexpr(kProf) count_block(ctx, 14, 7u);
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r37, R.r40, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, R.r41, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r39, R.r42, bitcast<float>(R.r14))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r53)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r53)) > static_cast<float>((0x0.0p+0f))));
        goto L_B15;
    L_B15: // isect_triangle_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 15, 7u);
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r53)) < static_cast<float>(R.r31))));
        R.r31 = static_cast<float>(((R.r49) ? (bitcast<float>(R.r53)) : (R.r31)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r33) + static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r32 = static_cast<unsigned int>(((R.r49) ? (R.r10) : (R.r32)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r33) == static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r33 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r33) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        if(R.r14) goto L_B16; else goto L_B11;
    L_B16: // traverse_sphere
        if(stop_heavy && !fresh) return 16;
    L_B16_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 16, 25u);
        R.r28 = static_cast<float>((0x1.99999a0000000p-4f));
        R.r29 = static_cast<float>((-0x1.6666660000000p-1f));
        R.r30 = static_cast<float>((0x1.3333340000000p-2f));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r20) - static_cast<float>(R.r28)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r21) - static_cast<float>(R.r29)));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r30)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.3333340000000p-2f)) * static_cast<float>((0x1.3333340000000p-2f)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r37, R.r37, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, R.r38, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r39, R.r39, bitcast<float>(R.r10))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) - static_cast<float>(bitcast<float>(R.r14))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r39) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r35 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r35 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r37, bitcast<float>(R.r35))));
        R.r35 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r38, bitcast<float>(R.r35))));
        R.r35 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r27, R.r39, bitcast<float>(R.r35))));
        R.r34 = static_cast<float>((0x0.0p+0f));
        R.r34 = static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), R.r34));
        R.r34 = static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), R.r34));
        R.r34 = static_cast<float>(op_fma(R.r27, R.r27, R.r34));
        R.r33 = static_cast<unsigned int>(((unsigned int)0x8ull));
        goto L_B17;
    L_B17: // traverse_solve_quadratic
        if(budget == 0u) return 17;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 17, 3u);
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(R.r34))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r49)) > static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r49) goto L_B20; else goto L_B18;
    L_B18: // sq_head1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 18, 3u);
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r35)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r49)) > static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r49) goto L_B19; else goto L_B24;
    L_B19: // sq_head2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 19, 3u);
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(-static_cast<float>(R.r36))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r53)) / static_cast<float>(bitcast<float>(R.r35)))));
        goto L_B24;
    L_B20: // sq_mid1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 20, 5u);
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(R.r34))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>((0x1.0000000000000p+2f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r35), bitcast<float>(R.r35), (-(bitcast<float>(R.r14))))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r49) goto L_B21; else goto L_B24;
    L_B21: // sq_mid2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 21, 11u);
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r53 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r35)) < static_cast<float>((0x0.0p+0f))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r35)) - static_cast<float>(bitcast<float>(R.r49)))));
        R.r35 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r35)) + static_cast<float>(bitcast<float>(R.r49)))));
        R.r35 = bitcast<unsigned int>(static_cast<float>(((R.r53) ? (bitcast<float>(R.r10)) : (bitcast<float>(R.r35)))));
        R.r35 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r35)) * static_cast<float>((-0x1.0000000000000p-1f)))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r35)) / static_cast<float>(R.r34))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) / static_cast<float>(bitcast<float>(R.r35))));
        R.r35 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r53)) < static_cast<float>((0x0.0p+0f))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(((R.r35) ? (R.r36) : (bitcast<float>(R.r53)))));
        if(R.r35) goto L_B23; else goto L_B22;
    L_B22: // sq_mid
        fresh = false;
        if constexpr(kProf) count_block(ctx, 22, 4u);
        R.r35 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r36) < static_cast<float>((0x0.0p+0f))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_min<float>(static_cast<float>(bitcast<float>(R.r53)), static_cast<float>(R.r36))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(((R.r35) ? (bitcast<float>(R.r53)) : (bitcast<float>(R.r49)))));
        goto L_B23;
    L_B23: // sq_tail
        fresh = false;
        if constexpr(kProf) count_block(ctx, 23, 3u);
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r53)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r49)) >= static_cast<float>((0x0.0p+0f))));
        goto L_B24;
    L_B24: // sq_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 24, 2u);
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r33) == static_cast<unsigned int>(((unsigned int)0x8ull))));
        if(R.r14) goto L_B25; else goto L_B27;
    L_B25: // traverse_sphere_fin
        fresh = false;
        if constexpr(kProf) count_block(ctx, 25, 4u);
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r53)) < static_cast<float>(R.r31))));
        R.r31 = static_cast<float>(((R.r49) ? (bitcast<float>(R.r53)) : (R.r31)));
        R.r32 = static_cast<unsigned int>(((R.r49) ? (R.r33) : (R.r32)));
        goto L_B26;
    L_B26: // traverse_cylinder
        fresh = false;
        if constexpr(kProf) count_block(ctx, 26, 13u);
        R.r28 = static_cast<float>(static_cast<float>(static_cast<float>(R.r20) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r29 = static_cast<float>(static_cast<float>(static_cast<float>(R.r21) - static_cast<float>((-0x1.0000000000000p+0f))));
        R.r30 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>((-0x1.3333340000000p-2f))));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r27)));
        R.r34 = static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), R.r34));
        R.r35 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r30) * static_cast<float>(R.r27))));
        R.r35 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r28, bitcast<float>(R.r6), bitcast<float>(R.r35))));
        R.r35 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r35)) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p-2f)) * static_cast<float>((0x1.0000000000000p-2f))));
        R.r36 = static_cast<float>(op_fma(R.r30, R.r30, (-(R.r36))));
        R.r36 = static_cast<float>(op_fma(R.r28, R.r28, R.r36));
        R.r33 = static_cast<unsigned int>(((unsigned int)0x9ull));
        goto L_B17;
    L_B27: // traverse_cylinder_fin
        fresh = false;
        if constexpr(kProf) count_block(ctx, 27, 15u);
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r53), R.r29)));
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x0.0p+0f)))));
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) <= static_cast<float>((0x1.4ccccc0000000p-1f)))));
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r53)) < static_cast<float>(R.r31))));
        R.r31 = static_cast<float>(((R.r49) ? (bitcast<float>(R.r53)) : (R.r31)));
        R.r32 = static_cast<unsigned int>(((R.r49) ? (R.r33) : (R.r32)));
        R.r33 = static_cast<unsigned int>(((unsigned int)0xaull));
        R.r28 = static_cast<float>((0x1.0000000000000p-1f));
        R.r29 = static_cast<float>((-0x1.6666660000000p-2f));
        R.r30 = static_cast<float>((-0x1.3333340000000p-2f));
        R.r34 = static_cast<float>((0x0.0p+0f));
        R.r35 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p+0f)));
        R.r36 = static_cast<float>((0x0.0p+0f));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p-2f)));
        goto L_B28;
    L_B28: // traverse_disk
        if(budget == 0u) return 28;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 28, 14u);
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r28) - static_cast<float>(R.r20)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r29) - static_cast<float>(R.r21)));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r30) - static_cast<float>(R.r22)));
        R.r53 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r37, R.r34, bitcast<float>(R.r53))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, bitcast<float>(R.r35), bitcast<float>(R.r53))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r39, R.r36, bitcast<float>(R.r53))));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r34, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r35), bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r27, R.r36, bitcast<float>(R.r10))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r53)) / static_cast<float>(bitcast<float>(R.r10)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r53)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r49) goto L_B29; else goto L_B30;
    L_B29: // isect_disk_rest
        fresh = false;
        if constexpr(kProf) count_block(ctx, 29, 16u);
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r53))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r53))));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(bitcast<float>(R.r53))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) + static_cast<float>(R.r20)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) + static_cast<float>(R.r21)));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r39) + static_cast<float>(R.r22)));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) - static_cast<float>(R.r28)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) - static_cast<float>(R.r29)));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r39) - static_cast<float>(R.r30)));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r37, R.r37, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, R.r38, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r39, R.r39, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r10)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r10)) < static_cast<float>(bitcast<float>(R.r14))));
        goto L_B30;
    L_B30: // isect_disk_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 30, 13u);
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r53)) < static_cast<float>(R.r31))));
        R.r31 = static_cast<float>(((R.r49) ? (bitcast<float>(R.r53)) : (R.r31)));
        R.r32 = static_cast<unsigned int>(((R.r49) ? (R.r33) : (R.r32)));
        R.r10 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r33) == static_cast<unsigned int>(((unsigned int)0xbull))));
        R.r33 = static_cast<unsigned int>(((unsigned int)0xbull));
        R.r28 = static_cast<float>((0x0.0p+0f));
        R.r29 = static_cast<float>((0x1.fff2e40000000p-1f));
        R.r30 = static_cast<float>((0x0.0p+0f));
        R.r34 = static_cast<float>((0x0.0p+0f));
        R.r35 = bitcast<unsigned int>(static_cast<float>((-0x1.0000000000000p+0f)));
        R.r36 = static_cast<float>((0x0.0p+0f));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x1.6666660000000p-2f)));
        if(R.r10) goto L_B31; else goto L_B28;
    L_B31: // traverse_room_end
        if(stop_heavy && !fresh) return 31;
    L_B31_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 31, 20u);
        R.r5 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r5) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r14 = static_cast<unsigned int>(op_min<unsigned int>(static_cast<unsigned int>(R.r32), static_cast<unsigned int>(((unsigned int)0x7ull))));
        R.r23 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.99999a0000000p-1f) : ((R.r14) == 1 ? (0x1.0000000000000p+0f) : ((R.r14) == 2 ? (0x1.99999a0000000p-3f) : ((R.r14) == 3 ? (0x1.99999a0000000p-1f) : ((R.r14) == 4 ? (0x1.3333340000000p-2f) : ((R.r14) == 5 ? (0x0.0p+0f) : ((R.r14) == 6 ? (0x0.0p+0f) : (0x0.0p+0f))))))))));
        R.r24 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.99999a0000000p-1f) : ((R.r14) == 1 ? (0x1.99999a0000000p-2f) : ((R.r14) == 2 ? (0x1.0000000000000p+0f) : ((R.r14) == 3 ? (0x1.99999a0000000p-1f) : ((R.r14) == 4 ? (0x1.99999a0000000p-2f) : ((R.r14) == 5 ? (0x1.b22d100000000p-3f) : ((R.r14) == 6 ? (0x1.b22d100000000p-3f) : (0x1.b22d100000000p-3f))))))))));
        R.r25 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.99999a0000000p-1f) : ((R.r14) == 1 ? (0x1.99999a0000000p-3f) : ((R.r14) == 2 ? (0x1.99999a0000000p-2f) : ((R.r14) == 3 ? (0x1.99999a0000000p-1f) : ((R.r14) == 4 ? (0x1.99999a0000000p-2f) : ((R.r14) == 5 ? (0x1.1b22d20000000p-1f) : ((R.r14) == 6 ? (0x1.1b22d20000000p-1f) : (0x1.1b22d20000000p-1f))))))))));
        R.r14 = static_cast<unsigned int>(op_max<unsigned int>(static_cast<unsigned int>(R.r32), static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r14 = static_cast<unsigned int>(op_min<unsigned int>(static_cast<unsigned int>(R.r14), static_cast<unsigned int>(((unsigned int)0xbull))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) - static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r28 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.99999a0000000p-1f) : ((R.r14) == 1 ? (0x1.0000000000000p+0f) : ((R.r14) == 2 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f))))));
        R.r29 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.99999a0000000p-3f) : ((R.r14) == 1 ? (0x1.926e980000000p-1f) : ((R.r14) == 2 ? (0x1.926e980000000p-1f) : (0x1.0000000000000p+0f))))));
        R.r30 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.99999a0000000p-1f) : ((R.r14) == 1 ? (0x1.b53f7e0000000p-2f) : ((R.r14) == 2 ? (0x1.b53f7e0000000p-2f) : (0x1.0000000000000p+0f))))));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r32) <= static_cast<unsigned int>(((unsigned int)0x7ull))));
        R.r23 = static_cast<float>(((R.r14) ? (R.r23) : (R.r28)));
        R.r24 = static_cast<float>(((R.r14) ? (R.r24) : (R.r29)));
        R.r25 = static_cast<float>(((R.r14) ? (R.r25) : (R.r30)));
        R.r2 = static_cast<float>(static_cast<float>(static_cast<float>(R.r2) + static_cast<float>(R.r23)));
        R.r3 = static_cast<float>(static_cast<float>(static_cast<float>(R.r3) + static_cast<float>(R.r24)));
        R.r4 = static_cast<float>(static_cast<float>(static_cast<float>(R.r4) + static_cast<float>(R.r25)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r17) >= static_cast<unsigned int>(((unsigned int)0x40ull))));
        if(R.r14) goto L_B32; else goto L_B1;
    L_B32: // fin_pixel
        fresh = false;
        if constexpr(kProf) count_block(ctx, 32, 4u);
        R.r2 = static_cast<float>(static_cast<float>(static_cast<float>(R.r2) / static_cast<float>((0x1.0000000000000p+6f))));
        R.r3 = static_cast<float>(static_cast<float>(static_cast<float>(R.r3) / static_cast<float>((0x1.0000000000000p+6f))));
        R.r4 = static_cast<float>(static_cast<float>(static_cast<float>(R.r4) / static_cast<float>((0x1.0000000000000p+6f))));
        goto L_HALT;
    L_HALT:
        return kHalt;
    }

    static constexpr unsigned long long kRowBytes = 3416ull;
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
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r53);
                v0.z = tid;
                reinterpret_cast<uint4*>(base + 0ull * cap)[idx] = v0;
            }
            return;
        }
        case 1: // roll
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 16ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r8);
                v1.z = bitcast<unsigned>(R.r9);
                v1.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 32ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r13);
                v2.y = bitcast<unsigned>(R.r15);
                v2.z = bitcast<unsigned>(R.r17);
                v2.w = bitcast<unsigned>(R.r53);
                reinterpret_cast<uint4*>(base + 48ull * cap)[idx] = v2;
            }
            {
                unsigned v3;
                v3 = tid;
                reinterpret_cast<unsigned*>(base + 64ull * cap)[idx] = v3;
            }
            return;
        }
        case 2: // traverse_box
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 72ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 88ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 104ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 120ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r31);
                v4.z = bitcast<unsigned>(R.r32);
                v4.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 136ull * cap)[idx] = v4;
            }
            {
                uint2 v5;
                v5.x = bitcast<unsigned>(R.r53);
                v5.y = tid;
                reinterpret_cast<uint2*>(base + 152ull * cap)[idx] = v5;
            }
            return;
        }
        case 3: // isect_quad_l1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 160ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 176ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 192ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 208ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r28);
                v4.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 224ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r30);
                v5.y = bitcast<unsigned>(R.r31);
                v5.z = bitcast<unsigned>(R.r32);
                v5.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 240ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r34);
                v6.y = bitcast<unsigned>(R.r35);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 256ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r39);
                v7.z = bitcast<unsigned>(R.r40);
                v7.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 272ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r42);
                v8.y = bitcast<unsigned>(R.r50);
                v8.z = bitcast<unsigned>(R.r51);
                v8.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 288ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r53);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 304ull * cap)[idx] = v9;
            }
            return;
        }
        case 4: // isect_quad_l2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 312ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 328ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r10);
                v2.z = bitcast<unsigned>(R.r12);
                v2.w = bitcast<unsigned>(R.r13);
                reinterpret_cast<uint4*>(base + 344ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r14);
                v3.y = bitcast<unsigned>(R.r15);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r20);
                reinterpret_cast<uint4*>(base + 360ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r21);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r27);
                v4.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 376ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r29);
                v5.y = bitcast<unsigned>(R.r30);
                v5.z = bitcast<unsigned>(R.r31);
                v5.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 392ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r33);
                v6.y = bitcast<unsigned>(R.r34);
                v6.z = bitcast<unsigned>(R.r35);
                v6.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 408ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r37);
                v7.y = bitcast<unsigned>(R.r38);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 424ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r42);
                v8.z = bitcast<unsigned>(R.r53);
                v8.w = tid;
                reinterpret_cast<uint4*>(base + 440ull * cap)[idx] = v8;
            }
            return;
        }
        case 5: // isect_quad_l3
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 456ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 472ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r10);
                v2.z = bitcast<unsigned>(R.r11);
                v2.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 488ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r13);
                v3.y = bitcast<unsigned>(R.r14);
                v3.z = bitcast<unsigned>(R.r15);
                v3.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 504ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r20);
                v4.y = bitcast<unsigned>(R.r21);
                v4.z = bitcast<unsigned>(R.r22);
                v4.w = bitcast<unsigned>(R.r27);
                reinterpret_cast<uint4*>(base + 520ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r28);
                v5.y = bitcast<unsigned>(R.r29);
                v5.z = bitcast<unsigned>(R.r30);
                v5.w = bitcast<unsigned>(R.r31);
                reinterpret_cast<uint4*>(base + 536ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r32);
                v6.y = bitcast<unsigned>(R.r33);
                v6.z = bitcast<unsigned>(R.r34);
                v6.w = bitcast<unsigned>(R.r35);
                reinterpret_cast<uint4*>(base + 552ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r36);
                v7.y = bitcast<unsigned>(R.r37);
                v7.z = bitcast<unsigned>(R.r38);
                v7.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 568ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r40);
                v8.y = bitcast<unsigned>(R.r41);
                v8.z = bitcast<unsigned>(R.r42);
                v8.w = tid;
                reinterpret_cast<uint4*>(base + 584ull * cap)[idx] = v8;
            }
            return;
        }
        case 6: // isect_quad_l4
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 600ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 616ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 632ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 648ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r28);
                v4.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 664ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r30);
                v5.y = bitcast<unsigned>(R.r31);
                v5.z = bitcast<unsigned>(R.r32);
                v5.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 680ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r34);
                v6.y = bitcast<unsigned>(R.r35);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 696ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r39);
                v7.z = bitcast<unsigned>(R.r40);
                v7.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 712ull * cap)[idx] = v7;
            }
            {
                uint2 v8;
                v8.x = bitcast<unsigned>(R.r42);
                v8.y = tid;
                reinterpret_cast<uint2*>(base + 728ull * cap)[idx] = v8;
            }
            return;
        }
        case 7: // isect_quad_l5
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 736ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 752ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 768ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 784ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r28);
                v4.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 800ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r30);
                v5.y = bitcast<unsigned>(R.r31);
                v5.z = bitcast<unsigned>(R.r32);
                v5.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 816ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r34);
                v6.y = bitcast<unsigned>(R.r35);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 832ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r39);
                v7.z = bitcast<unsigned>(R.r40);
                v7.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 848ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r42);
                v8.y = bitcast<unsigned>(R.r43);
                v8.z = bitcast<unsigned>(R.r44);
                v8.w = bitcast<unsigned>(R.r45);
                reinterpret_cast<uint4*>(base + 864ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r50);
                v9.y = bitcast<unsigned>(R.r51);
                v9.z = bitcast<unsigned>(R.r52);
                v9.w = bitcast<unsigned>(R.r53);
                reinterpret_cast<uint4*>(base + 880ull * cap)[idx] = v9;
            }
            {
                unsigned v10;
                v10 = tid;
                reinterpret_cast<unsigned*>(base + 896ull * cap)[idx] = v10;
            }
            return;
        }
        case 8: // isect_quad_l6
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 904ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 920ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 936ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 952ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r28);
                v4.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 968ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r30);
                v5.y = bitcast<unsigned>(R.r31);
                v5.z = bitcast<unsigned>(R.r32);
                v5.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 984ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r34);
                v6.y = bitcast<unsigned>(R.r35);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 1000ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r41);
                v7.y = bitcast<unsigned>(R.r42);
                v7.z = bitcast<unsigned>(R.r43);
                v7.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 1016ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r45);
                v8.y = bitcast<unsigned>(R.r46);
                v8.z = bitcast<unsigned>(R.r47);
                v8.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 1032ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r53);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 1048ull * cap)[idx] = v9;
            }
            return;
        }
        case 9: // isect_quad_l7
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1056ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1072ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 1088ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 1104ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r28);
                v4.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 1120ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r30);
                v5.y = bitcast<unsigned>(R.r31);
                v5.z = bitcast<unsigned>(R.r32);
                v5.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1136ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r34);
                v6.y = bitcast<unsigned>(R.r35);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 1152ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r41);
                v7.y = bitcast<unsigned>(R.r42);
                v7.z = tid;
                reinterpret_cast<uint4*>(base + 1168ull * cap)[idx] = v7;
            }
            return;
        }
        case 10: // isect_quad_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1184ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1200ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 1216ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 1232ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r31);
                v4.z = bitcast<unsigned>(R.r32);
                v4.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1248ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r49);
                v5.y = bitcast<unsigned>(R.r53);
                v5.z = tid;
                reinterpret_cast<uint4*>(base + 1264ull * cap)[idx] = v5;
            }
            return;
        }
        case 11: // traverse_tetrahedron
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1280ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1296ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 1312ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 1328ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r31);
                v4.z = bitcast<unsigned>(R.r32);
                v4.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1344ull * cap)[idx] = v4;
            }
            {
                unsigned v5;
                v5 = tid;
                reinterpret_cast<unsigned*>(base + 1360ull * cap)[idx] = v5;
            }
            return;
        }
        case 12: // isect_triangle_mid1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1368ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1384ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 1400ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 1416ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r28);
                v4.z = bitcast<unsigned>(R.r29);
                v4.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 1432ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r31);
                v5.y = bitcast<unsigned>(R.r32);
                v5.z = bitcast<unsigned>(R.r33);
                v5.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 1448ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r35);
                v6.y = bitcast<unsigned>(R.r36);
                v6.z = bitcast<unsigned>(R.r37);
                v6.w = bitcast<unsigned>(R.r38);
                reinterpret_cast<uint4*>(base + 1464ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r39);
                v7.y = bitcast<unsigned>(R.r40);
                v7.z = bitcast<unsigned>(R.r41);
                v7.w = bitcast<unsigned>(R.r42);
                reinterpret_cast<uint4*>(base + 1480ull * cap)[idx] = v7;
            }
            {
                uint2 v8;
                v8.x = bitcast<unsigned>(R.r53);
                v8.y = tid;
                reinterpret_cast<uint2*>(base + 1496ull * cap)[idx] = v8;
            }
            return;
        }
        case 13: // isect_triangle_mid2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1504ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1520ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 1536ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 1552ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r28);
                v4.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 1568ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r30);
                v5.y = bitcast<unsigned>(R.r31);
                v5.z = bitcast<unsigned>(R.r32);
                v5.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1584ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r34);
                v6.y = bitcast<unsigned>(R.r35);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 1600ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r39);
                v7.z = bitcast<unsigned>(R.r53);
                v7.w = tid;
                reinterpret_cast<uint4*>(base + 1616ull * cap)[idx] = v7;
            }
            return;
        }
        case 14: // isect_triangle_mid3
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1632ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1648ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 1664ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 1680ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r31);
                v4.z = bitcast<unsigned>(R.r32);
                v4.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1696ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r37);
                v5.y = bitcast<unsigned>(R.r38);
                v5.z = bitcast<unsigned>(R.r39);
                v5.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 1712ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r41);
                v6.y = bitcast<unsigned>(R.r42);
                v6.z = bitcast<unsigned>(R.r53);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 1728ull * cap)[idx] = v6;
            }
            return;
        }
        case 15: // isect_triangle_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1744ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1760ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 1776ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 1792ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r31);
                v4.z = bitcast<unsigned>(R.r32);
                v4.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1808ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r49);
                v5.y = bitcast<unsigned>(R.r53);
                v5.z = tid;
                reinterpret_cast<uint4*>(base + 1824ull * cap)[idx] = v5;
            }
            return;
        }
        case 16: // traverse_sphere
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1840ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1856ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 1872ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 1888ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r31);
                v4.z = bitcast<unsigned>(R.r32);
                v4.w = bitcast<unsigned>(R.r53);
                reinterpret_cast<uint4*>(base + 1904ull * cap)[idx] = v4;
            }
            {
                unsigned v5;
                v5 = tid;
                reinterpret_cast<unsigned*>(base + 1920ull * cap)[idx] = v5;
            }
            return;
        }
        case 17: // traverse_solve_quadratic
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1928ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1944ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 1960ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 1976ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r29);
                v4.z = bitcast<unsigned>(R.r31);
                v4.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 1992ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r33);
                v5.y = bitcast<unsigned>(R.r34);
                v5.z = bitcast<unsigned>(R.r35);
                v5.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 2008ull * cap)[idx] = v5;
            }
            {
                uint2 v6;
                v6.x = bitcast<unsigned>(R.r53);
                v6.y = tid;
                reinterpret_cast<uint2*>(base + 2024ull * cap)[idx] = v6;
            }
            return;
        }
        case 18: // sq_head1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2032ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2048ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2064ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2080ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r29);
                v4.z = bitcast<unsigned>(R.r31);
                v4.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 2096ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r33);
                v5.y = bitcast<unsigned>(R.r35);
                v5.z = bitcast<unsigned>(R.r36);
                v5.w = bitcast<unsigned>(R.r53);
                reinterpret_cast<uint4*>(base + 2112ull * cap)[idx] = v5;
            }
            {
                unsigned v6;
                v6 = tid;
                reinterpret_cast<unsigned*>(base + 2128ull * cap)[idx] = v6;
            }
            return;
        }
        case 19: // sq_head2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2136ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2152ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2168ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2184ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r29);
                v4.z = bitcast<unsigned>(R.r31);
                v4.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 2200ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r33);
                v5.y = bitcast<unsigned>(R.r35);
                v5.z = bitcast<unsigned>(R.r36);
                v5.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 2216ull * cap)[idx] = v5;
            }
            {
                unsigned v6;
                v6 = tid;
                reinterpret_cast<unsigned*>(base + 2232ull * cap)[idx] = v6;
            }
            return;
        }
        case 20: // sq_mid1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2240ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2256ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2272ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2288ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r29);
                v4.z = bitcast<unsigned>(R.r31);
                v4.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 2304ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r33);
                v5.y = bitcast<unsigned>(R.r34);
                v5.z = bitcast<unsigned>(R.r35);
                v5.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 2320ull * cap)[idx] = v5;
            }
            {
                uint2 v6;
                v6.x = bitcast<unsigned>(R.r53);
                v6.y = tid;
                reinterpret_cast<uint2*>(base + 2336ull * cap)[idx] = v6;
            }
            return;
        }
        case 21: // sq_mid2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2344ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2360ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 2376ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 2392ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r29);
                v4.w = bitcast<unsigned>(R.r31);
                reinterpret_cast<uint4*>(base + 2408ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r32);
                v5.y = bitcast<unsigned>(R.r33);
                v5.z = bitcast<unsigned>(R.r34);
                v5.w = bitcast<unsigned>(R.r35);
                reinterpret_cast<uint4*>(base + 2424ull * cap)[idx] = v5;
            }
            {
                uint2 v6;
                v6.x = bitcast<unsigned>(R.r36);
                v6.y = tid;
                reinterpret_cast<uint2*>(base + 2440ull * cap)[idx] = v6;
            }
            return;
        }
        case 22: // sq_mid
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2448ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2464ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 2480ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 2496ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r29);
                v4.w = bitcast<unsigned>(R.r31);
                reinterpret_cast<uint4*>(base + 2512ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r32);
                v5.y = bitcast<unsigned>(R.r33);
                v5.z = bitcast<unsigned>(R.r36);
                v5.w = bitcast<unsigned>(R.r53);
                reinterpret_cast<uint4*>(base + 2528ull * cap)[idx] = v5;
            }
            {
                unsigned v6;
                v6 = tid;
                reinterpret_cast<unsigned*>(base + 2544ull * cap)[idx] = v6;
            }
            return;
        }
        case 23: // sq_tail
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2552ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2568ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 2584ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 2600ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r29);
                v4.w = bitcast<unsigned>(R.r31);
                reinterpret_cast<uint4*>(base + 2616ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r32);
                v5.y = bitcast<unsigned>(R.r33);
                v5.z = bitcast<unsigned>(R.r53);
                v5.w = tid;
                reinterpret_cast<uint4*>(base + 2632ull * cap)[idx] = v5;
            }
            return;
        }
        case 24: // sq_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2648ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2664ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2680ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2696ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r29);
                v4.z = bitcast<unsigned>(R.r31);
                v4.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 2712ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r33);
                v5.y = bitcast<unsigned>(R.r49);
                v5.z = bitcast<unsigned>(R.r53);
                v5.w = tid;
                reinterpret_cast<uint4*>(base + 2728ull * cap)[idx] = v5;
            }
            return;
        }
        case 25: // traverse_sphere_fin
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2744ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2760ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2776ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2792ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r31);
                v4.z = bitcast<unsigned>(R.r32);
                v4.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 2808ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r49);
                v5.y = bitcast<unsigned>(R.r53);
                v5.z = tid;
                reinterpret_cast<uint4*>(base + 2824ull * cap)[idx] = v5;
            }
            return;
        }
        case 26: // traverse_cylinder
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2840ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2856ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2872ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2888ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r31);
                v4.z = bitcast<unsigned>(R.r32);
                v4.w = bitcast<unsigned>(R.r53);
                reinterpret_cast<uint4*>(base + 2904ull * cap)[idx] = v4;
            }
            {
                unsigned v5;
                v5 = tid;
                reinterpret_cast<unsigned*>(base + 2920ull * cap)[idx] = v5;
            }
            return;
        }
        case 27: // traverse_cylinder_fin
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2928ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2944ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2960ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2976ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r29);
                v4.z = bitcast<unsigned>(R.r31);
                v4.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 2992ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r33);
                v5.y = bitcast<unsigned>(R.r49);
                v5.z = bitcast<unsigned>(R.r53);
                v5.w = tid;
                reinterpret_cast<uint4*>(base + 3008ull * cap)[idx] = v5;
            }
            return;
        }
        case 28: // traverse_disk
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3024ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 3040ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 3056ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 3072ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r28);
                v4.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 3088ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r30);
                v5.y = bitcast<unsigned>(R.r31);
                v5.z = bitcast<unsigned>(R.r32);
                v5.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 3104ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r34);
                v6.y = bitcast<unsigned>(R.r35);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 3120ull * cap)[idx] = v6;
            }
            return;
        }
        case 29: // isect_disk_rest
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3136ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 3152ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 3168ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 3184ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r27);
                v4.z = bitcast<unsigned>(R.r28);
                v4.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 3200ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r30);
                v5.y = bitcast<unsigned>(R.r31);
                v5.z = bitcast<unsigned>(R.r32);
                v5.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 3216ull * cap)[idx] = v5;
            }
            {
                uint2 v6;
                v6.x = bitcast<unsigned>(R.r53);
                v6.y = tid;
                reinterpret_cast<uint2*>(base + 3232ull * cap)[idx] = v6;
            }
            return;
        }
        case 30: // isect_disk_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3240ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 3256ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 3272ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r17);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 3288ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r27);
                v4.y = bitcast<unsigned>(R.r31);
                v4.z = bitcast<unsigned>(R.r32);
                v4.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 3304ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r49);
                v5.y = bitcast<unsigned>(R.r53);
                v5.z = tid;
                reinterpret_cast<uint4*>(base + 3320ull * cap)[idx] = v5;
            }
            return;
        }
        case 31: // traverse_room_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3336ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r8);
                v1.z = bitcast<unsigned>(R.r9);
                v1.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 3352ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r13);
                v2.y = bitcast<unsigned>(R.r15);
                v2.z = bitcast<unsigned>(R.r17);
                v2.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 3368ull * cap)[idx] = v2;
            }
            {
                uint2 v3;
                v3.x = bitcast<unsigned>(R.r53);
                v3.y = tid;
                reinterpret_cast<uint2*>(base + 3384ull * cap)[idx] = v3;
            }
            return;
        }
        case 32: // fin_pixel
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3392ull * cap)[idx] = v0;
            }
            {
                uint2 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = tid;
                reinterpret_cast<uint2*>(base + 3408ull * cap)[idx] = v1;
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
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 0ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r53 = bitcast<unsigned int>(v0.y);
            return v0.z;
        }
        case 1: // roll
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 16ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 32ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r8 = bitcast<unsigned int>(v1.y);
            R.r9 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 48ull * cap)[idx];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r17 = bitcast<unsigned int>(v2.z);
            R.r53 = bitcast<unsigned int>(v2.w);
            const unsigned v3 = reinterpret_cast<const unsigned*>(base + 64ull * cap)[idx];
            return v3;
        }
        case 2: // traverse_box
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 72ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 88ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 104ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 120ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 136ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint2 v5 = reinterpret_cast<const uint2*>(base + 152ull * cap)[idx];
            R.r53 = bitcast<unsigned int>(v5.x);
            return v5.y;
        }
        case 3: // isect_quad_l1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 160ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 176ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 192ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 208ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 224ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 240ull * cap)[idx];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 256ull * cap)[idx];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 272ull * cap)[idx];
            R.r38 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r40 = bitcast<float>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 288ull * cap)[idx];
            R.r42 = bitcast<float>(v8.x);
            R.r50 = bitcast<float>(v8.y);
            R.r51 = bitcast<float>(v8.z);
            R.r52 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 304ull * cap)[idx];
            R.r53 = bitcast<unsigned int>(v9.x);
            return v9.y;
        }
        case 4: // isect_quad_l2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 312ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 328ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 344ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r12 = bitcast<float>(v2.z);
            R.r13 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 360ull * cap)[idx];
            R.r14 = bitcast<unsigned int>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r17 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 376ull * cap)[idx];
            R.r21 = bitcast<float>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r27 = bitcast<float>(v4.z);
            R.r28 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 392ull * cap)[idx];
            R.r29 = bitcast<float>(v5.x);
            R.r30 = bitcast<float>(v5.y);
            R.r31 = bitcast<float>(v5.z);
            R.r32 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 408ull * cap)[idx];
            R.r33 = bitcast<unsigned int>(v6.x);
            R.r34 = bitcast<float>(v6.y);
            R.r35 = bitcast<unsigned int>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 424ull * cap)[idx];
            R.r37 = bitcast<float>(v7.x);
            R.r38 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 440ull * cap)[idx];
            R.r41 = bitcast<float>(v8.x);
            R.r42 = bitcast<float>(v8.y);
            R.r53 = bitcast<unsigned int>(v8.z);
            return v8.w;
        }
        case 5: // isect_quad_l3
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 456ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 472ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 488ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r11 = bitcast<unsigned int>(v2.z);
            R.r12 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 504ull * cap)[idx];
            R.r13 = bitcast<float>(v3.x);
            R.r14 = bitcast<unsigned int>(v3.y);
            R.r15 = bitcast<float>(v3.z);
            R.r17 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 520ull * cap)[idx];
            R.r20 = bitcast<float>(v4.x);
            R.r21 = bitcast<float>(v4.y);
            R.r22 = bitcast<float>(v4.z);
            R.r27 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 536ull * cap)[idx];
            R.r28 = bitcast<float>(v5.x);
            R.r29 = bitcast<float>(v5.y);
            R.r30 = bitcast<float>(v5.z);
            R.r31 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 552ull * cap)[idx];
            R.r32 = bitcast<unsigned int>(v6.x);
            R.r33 = bitcast<unsigned int>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r35 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 568ull * cap)[idx];
            R.r36 = bitcast<float>(v7.x);
            R.r37 = bitcast<float>(v7.y);
            R.r38 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 584ull * cap)[idx];
            R.r40 = bitcast<float>(v8.x);
            R.r41 = bitcast<float>(v8.y);
            R.r42 = bitcast<float>(v8.z);
            return v8.w;
        }
        case 6: // isect_quad_l4
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 600ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 616ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 632ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 648ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 664ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 680ull * cap)[idx];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 696ull * cap)[idx];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 712ull * cap)[idx];
            R.r38 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r40 = bitcast<float>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint2 v8 = reinterpret_cast<const uint2*>(base + 728ull * cap)[idx];
            R.r42 = bitcast<float>(v8.x);
            return v8.y;
        }
        case 7: // isect_quad_l5
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 736ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 752ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 768ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 784ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 800ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 816ull * cap)[idx];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 832ull * cap)[idx];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 848ull * cap)[idx];
            R.r38 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r40 = bitcast<float>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 864ull * cap)[idx];
            R.r42 = bitcast<float>(v8.x);
            R.r43 = bitcast<float>(v8.y);
            R.r44 = bitcast<float>(v8.z);
            R.r45 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 880ull * cap)[idx];
            R.r50 = bitcast<float>(v9.x);
            R.r51 = bitcast<float>(v9.y);
            R.r52 = bitcast<float>(v9.z);
            R.r53 = bitcast<unsigned int>(v9.w);
            const unsigned v10 = reinterpret_cast<const unsigned*>(base + 896ull * cap)[idx];
            return v10;
        }
        case 8: // isect_quad_l6
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 904ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 920ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 936ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 952ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 968ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 984ull * cap)[idx];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1000ull * cap)[idx];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r40 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1016ull * cap)[idx];
            R.r41 = bitcast<float>(v7.x);
            R.r42 = bitcast<float>(v7.y);
            R.r43 = bitcast<float>(v7.z);
            R.r44 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1032ull * cap)[idx];
            R.r45 = bitcast<float>(v8.x);
            R.r46 = bitcast<float>(v8.y);
            R.r47 = bitcast<float>(v8.z);
            R.r48 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 1048ull * cap)[idx];
            R.r53 = bitcast<unsigned int>(v9.x);
            return v9.y;
        }
        case 9: // isect_quad_l7
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1056ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1072ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1088ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1104ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1120ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1136ull * cap)[idx];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1152ull * cap)[idx];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r40 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1168ull * cap)[idx];
            R.r41 = bitcast<float>(v7.x);
            R.r42 = bitcast<float>(v7.y);
            return v7.z;
        }
        case 10: // isect_quad_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1184ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1200ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1216ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1232ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1248ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1264ull * cap)[idx];
            R.r49 = bitcast<unsigned int>(v5.x);
            R.r53 = bitcast<unsigned int>(v5.y);
            return v5.z;
        }
        case 11: // traverse_tetrahedron
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1280ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1296ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1312ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1328ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1344ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const unsigned v5 = reinterpret_cast<const unsigned*>(base + 1360ull * cap)[idx];
            return v5;
        }
        case 12: // isect_triangle_mid1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1368ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1384ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1400ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1416ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1432ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r28 = bitcast<float>(v4.y);
            R.r29 = bitcast<float>(v4.z);
            R.r30 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1448ull * cap)[idx];
            R.r31 = bitcast<float>(v5.x);
            R.r32 = bitcast<unsigned int>(v5.y);
            R.r33 = bitcast<unsigned int>(v5.z);
            R.r34 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1464ull * cap)[idx];
            R.r35 = bitcast<unsigned int>(v6.x);
            R.r36 = bitcast<float>(v6.y);
            R.r37 = bitcast<float>(v6.z);
            R.r38 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1480ull * cap)[idx];
            R.r39 = bitcast<float>(v7.x);
            R.r40 = bitcast<float>(v7.y);
            R.r41 = bitcast<float>(v7.z);
            R.r42 = bitcast<float>(v7.w);
            const uint2 v8 = reinterpret_cast<const uint2*>(base + 1496ull * cap)[idx];
            R.r53 = bitcast<unsigned int>(v8.x);
            return v8.y;
        }
        case 13: // isect_triangle_mid2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1504ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1520ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1536ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1552ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1568ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1584ull * cap)[idx];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1600ull * cap)[idx];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1616ull * cap)[idx];
            R.r38 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r53 = bitcast<unsigned int>(v7.z);
            return v7.w;
        }
        case 14: // isect_triangle_mid3
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1632ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1648ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1664ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1680ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1696ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1712ull * cap)[idx];
            R.r37 = bitcast<float>(v5.x);
            R.r38 = bitcast<float>(v5.y);
            R.r39 = bitcast<float>(v5.z);
            R.r40 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1728ull * cap)[idx];
            R.r41 = bitcast<float>(v6.x);
            R.r42 = bitcast<float>(v6.y);
            R.r53 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 15: // isect_triangle_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1744ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1760ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1776ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1792ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1808ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1824ull * cap)[idx];
            R.r49 = bitcast<unsigned int>(v5.x);
            R.r53 = bitcast<unsigned int>(v5.y);
            return v5.z;
        }
        case 16: // traverse_sphere
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1840ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1856ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1872ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1888ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1904ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<unsigned int>(v4.w);
            const unsigned v5 = reinterpret_cast<const unsigned*>(base + 1920ull * cap)[idx];
            return v5;
        }
        case 17: // traverse_solve_quadratic
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1928ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1944ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1960ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1976ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1992ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2008ull * cap)[idx];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r34 = bitcast<float>(v5.y);
            R.r35 = bitcast<unsigned int>(v5.z);
            R.r36 = bitcast<float>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(base + 2024ull * cap)[idx];
            R.r53 = bitcast<unsigned int>(v6.x);
            return v6.y;
        }
        case 18: // sq_head1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2032ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2048ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2064ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2080ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2096ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2112ull * cap)[idx];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r35 = bitcast<unsigned int>(v5.y);
            R.r36 = bitcast<float>(v5.z);
            R.r53 = bitcast<unsigned int>(v5.w);
            const unsigned v6 = reinterpret_cast<const unsigned*>(base + 2128ull * cap)[idx];
            return v6;
        }
        case 19: // sq_head2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2136ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2152ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2168ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2184ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2200ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2216ull * cap)[idx];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r35 = bitcast<unsigned int>(v5.y);
            R.r36 = bitcast<float>(v5.z);
            R.r49 = bitcast<unsigned int>(v5.w);
            const unsigned v6 = reinterpret_cast<const unsigned*>(base + 2232ull * cap)[idx];
            return v6;
        }
        case 20: // sq_mid1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2240ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2256ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2272ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2288ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2304ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2320ull * cap)[idx];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r34 = bitcast<float>(v5.y);
            R.r35 = bitcast<unsigned int>(v5.z);
            R.r36 = bitcast<float>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(base + 2336ull * cap)[idx];
            R.r53 = bitcast<unsigned int>(v6.x);
            return v6.y;
        }
        case 21: // sq_mid2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2344ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2360ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2376ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2392ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2408ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r29 = bitcast<float>(v4.z);
            R.r31 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2424ull * cap)[idx];
            R.r32 = bitcast<unsigned int>(v5.x);
            R.r33 = bitcast<unsigned int>(v5.y);
            R.r34 = bitcast<float>(v5.z);
            R.r35 = bitcast<unsigned int>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(base + 2440ull * cap)[idx];
            R.r36 = bitcast<float>(v6.x);
            return v6.y;
        }
        case 22: // sq_mid
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2448ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2464ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2480ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2496ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2512ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r29 = bitcast<float>(v4.z);
            R.r31 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2528ull * cap)[idx];
            R.r32 = bitcast<unsigned int>(v5.x);
            R.r33 = bitcast<unsigned int>(v5.y);
            R.r36 = bitcast<float>(v5.z);
            R.r53 = bitcast<unsigned int>(v5.w);
            const unsigned v6 = reinterpret_cast<const unsigned*>(base + 2544ull * cap)[idx];
            return v6;
        }
        case 23: // sq_tail
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2552ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2568ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2584ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2600ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2616ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r29 = bitcast<float>(v4.z);
            R.r31 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2632ull * cap)[idx];
            R.r32 = bitcast<unsigned int>(v5.x);
            R.r33 = bitcast<unsigned int>(v5.y);
            R.r53 = bitcast<unsigned int>(v5.z);
            return v5.w;
        }
        case 24: // sq_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2648ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2664ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2680ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2696ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2712ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2728ull * cap)[idx];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r49 = bitcast<unsigned int>(v5.y);
            R.r53 = bitcast<unsigned int>(v5.z);
            return v5.w;
        }
        case 25: // traverse_sphere_fin
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2744ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2760ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2776ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2792ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2808ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2824ull * cap)[idx];
            R.r49 = bitcast<unsigned int>(v5.x);
            R.r53 = bitcast<unsigned int>(v5.y);
            return v5.z;
        }
        case 26: // traverse_cylinder
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2840ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2856ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2872ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2888ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2904ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<unsigned int>(v4.w);
            const unsigned v5 = reinterpret_cast<const unsigned*>(base + 2920ull * cap)[idx];
            return v5;
        }
        case 27: // traverse_cylinder_fin
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2928ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2944ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2960ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2976ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2992ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3008ull * cap)[idx];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r49 = bitcast<unsigned int>(v5.y);
            R.r53 = bitcast<unsigned int>(v5.z);
            return v5.w;
        }
        case 28: // traverse_disk
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3024ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3040ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3056ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3072ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3088ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3104ull * cap)[idx];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3120ull * cap)[idx];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 29: // isect_disk_rest
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3136ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3152ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3168ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3184ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3200ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3216ull * cap)[idx];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(base + 3232ull * cap)[idx];
            R.r53 = bitcast<unsigned int>(v6.x);
            return v6.y;
        }
        case 30: // isect_disk_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3240ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3256ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3272ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3288ull * cap)[idx];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3304ull * cap)[idx];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3320ull * cap)[idx];
            R.r49 = bitcast<unsigned int>(v5.x);
            R.r53 = bitcast<unsigned int>(v5.y);
            return v5.z;
        }
        case 31: // traverse_room_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3336ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3352ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r8 = bitcast<unsigned int>(v1.y);
            R.r9 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3368ull * cap)[idx];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r17 = bitcast<unsigned int>(v2.z);
            R.r32 = bitcast<unsigned int>(v2.w);
            const uint2 v3 = reinterpret_cast<const uint2*>(base + 3384ull * cap)[idx];
            R.r53 = bitcast<unsigned int>(v3.x);
            return v3.y;
        }
        case 32: // fin_pixel
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3392ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint2 v1 = reinterpret_cast<const uint2*>(base + 3408ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            return v1.y;
        }
        default: return 0xffffffffu;
        }
    }

    // bytes of one queue entry's slots, the largest over the queues
    static constexpr unsigned kMaxStageRow = 176u;
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
        case 0: bytes = 512u; break;
        case 1: bytes = 1664u; break;
        case 2: bytes = 2816u; break;
        case 3: bytes = 4864u; break;
        case 4: bytes = 4608u; break;
        case 5: bytes = 4608u; break;
        case 6: bytes = 4352u; break;
        case 7: bytes = 5248u; break;
        case 8: bytes = 4864u; break;
        case 9: bytes = 4096u; break;
        case 10: bytes = 3072u; break;
        case 11: bytes = 2688u; break;
        case 12: bytes = 4352u; break;
        case 13: bytes = 4096u; break;
        case 14: bytes = 3584u; break;
        case 15: bytes = 3072u; break;
        case 16: bytes = 2688u; break;
        case 17: bytes = 3328u; break;
        case 18: bytes = 3200u; break;
        case 19: bytes = 3200u; break;
        case 20: bytes = 3328u; break;
        case 21: bytes = 3328u; break;
        case 22: bytes = 3200u; break;
        case 23: bytes = 3072u; break;
        case 24: bytes = 3072u; break;
        case 25: bytes = 3072u; break;
        case 26: bytes = 2688u; break;
        case 27: bytes = 3072u; break;
        case 28: bytes = 3584u; break;
        case 29: bytes = 3328u; break;
        case 30: bytes = 3072u; break;
        case 31: bytes = 1792u; break;
        case 32: bytes = 768u; break;
        default: return false;
        }
        if((reinterpret_cast<unsigned long long>(base) | reinterpret_cast<unsigned long long>(stage)) & 15ull) return false;
        bulk_expect(mbar, bytes);
        switch(q)
        {
        case 0:
            bulk_copy(stage + 0u, base + 0ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 1:
            bulk_copy(stage + 0u, base + 16ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 32ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 48ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 64ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 2:
            bulk_copy(stage + 0u, base + 72ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 88ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 152ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 3:
            bulk_copy(stage + 0u, base + 160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 176ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 192ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 208ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 224ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 304ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 4:
            bulk_copy(stage + 0u, base + 312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 5:
            bulk_copy(stage + 0u, base + 456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 472ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 520ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 536ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 552ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 584ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 6:
            bulk_copy(stage + 0u, base + 600ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 616ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 632ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 648ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 664ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 680ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 728ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 7:
            bulk_copy(stage + 0u, base + 736ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 752ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 768ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 784ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 800ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 816ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 832ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 848ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 864ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 880ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 896ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 8:
            bulk_copy(stage + 0u, base + 904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 968ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1048ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 9:
            bulk_copy(stage + 0u, base + 1056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 10:
            bulk_copy(stage + 0u, base + 1184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 11:
            bulk_copy(stage + 0u, base + 1280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1360ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 12:
            bulk_copy(stage + 0u, base + 1368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1496ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 13:
            bulk_copy(stage + 0u, base + 1504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1520ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1536ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1552ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1584ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1600ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1616ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 14:
            bulk_copy(stage + 0u, base + 1632ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1648ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1664ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1680ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 15:
            bulk_copy(stage + 0u, base + 1744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 16:
            bulk_copy(stage + 0u, base + 1840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1920ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 17:
            bulk_copy(stage + 0u, base + 1928ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1944ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2024ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 18:
            bulk_copy(stage + 0u, base + 2032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2128ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 19:
            bulk_copy(stage + 0u, base + 2136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2232ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 20:
            bulk_copy(stage + 0u, base + 2240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2304ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2320ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2336ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 21:
            bulk_copy(stage + 0u, base + 2344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2440ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 22:
            bulk_copy(stage + 0u, base + 2448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2544ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 23:
            bulk_copy(stage + 0u, base + 2552ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2584ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2600ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2616ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2632ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 24:
            bulk_copy(stage + 0u, base + 2648ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2664ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2680ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 25:
            bulk_copy(stage + 0u, base + 2744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 26:
            bulk_copy(stage + 0u, base + 2840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2920ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 27:
            bulk_copy(stage + 0u, base + 2928ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2944ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 28:
            bulk_copy(stage + 0u, base + 3024ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3040ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 29:
            bulk_copy(stage + 0u, base + 3136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3232ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 30:
            bulk_copy(stage + 0u, base + 3240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3304ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3320ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 31:
            bulk_copy(stage + 0u, base + 3336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3384ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 32:
            bulk_copy(stage + 0u, base + 3392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3408ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
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
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r53 = bitcast<unsigned int>(v0.y);
            return v0.z;
        }
        case 1:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r8 = bitcast<unsigned int>(v1.y);
            R.r9 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r17 = bitcast<unsigned int>(v2.z);
            R.r53 = bitcast<unsigned int>(v2.w);
            const unsigned v3 = reinterpret_cast<const unsigned*>(stage + 1536u)[lane];
            return v3;
        }
        case 2:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint2 v5 = reinterpret_cast<const uint2*>(stage + 2560u)[lane];
            R.r53 = bitcast<unsigned int>(v5.x);
            return v5.y;
        }
        case 3:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r40 = bitcast<float>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r42 = bitcast<float>(v8.x);
            R.r50 = bitcast<float>(v8.y);
            R.r51 = bitcast<float>(v8.z);
            R.r52 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r53 = bitcast<unsigned int>(v9.x);
            return v9.y;
        }
        case 4:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r12 = bitcast<float>(v2.z);
            R.r13 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r14 = bitcast<unsigned int>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r17 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r21 = bitcast<float>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r27 = bitcast<float>(v4.z);
            R.r28 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r29 = bitcast<float>(v5.x);
            R.r30 = bitcast<float>(v5.y);
            R.r31 = bitcast<float>(v5.z);
            R.r32 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r33 = bitcast<unsigned int>(v6.x);
            R.r34 = bitcast<float>(v6.y);
            R.r35 = bitcast<unsigned int>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r37 = bitcast<float>(v7.x);
            R.r38 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<float>(v8.x);
            R.r42 = bitcast<float>(v8.y);
            R.r53 = bitcast<unsigned int>(v8.z);
            return v8.w;
        }
        case 5:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r11 = bitcast<unsigned int>(v2.z);
            R.r12 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r13 = bitcast<float>(v3.x);
            R.r14 = bitcast<unsigned int>(v3.y);
            R.r15 = bitcast<float>(v3.z);
            R.r17 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r20 = bitcast<float>(v4.x);
            R.r21 = bitcast<float>(v4.y);
            R.r22 = bitcast<float>(v4.z);
            R.r27 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r28 = bitcast<float>(v5.x);
            R.r29 = bitcast<float>(v5.y);
            R.r30 = bitcast<float>(v5.z);
            R.r31 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r32 = bitcast<unsigned int>(v6.x);
            R.r33 = bitcast<unsigned int>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r35 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r36 = bitcast<float>(v7.x);
            R.r37 = bitcast<float>(v7.y);
            R.r38 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r40 = bitcast<float>(v8.x);
            R.r41 = bitcast<float>(v8.y);
            R.r42 = bitcast<float>(v8.z);
            return v8.w;
        }
        case 6:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r40 = bitcast<float>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint2 v8 = reinterpret_cast<const uint2*>(stage + 4096u)[lane];
            R.r42 = bitcast<float>(v8.x);
            return v8.y;
        }
        case 7:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r40 = bitcast<float>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r42 = bitcast<float>(v8.x);
            R.r43 = bitcast<float>(v8.y);
            R.r44 = bitcast<float>(v8.z);
            R.r45 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r50 = bitcast<float>(v9.x);
            R.r51 = bitcast<float>(v9.y);
            R.r52 = bitcast<float>(v9.z);
            R.r53 = bitcast<unsigned int>(v9.w);
            const unsigned v10 = reinterpret_cast<const unsigned*>(stage + 5120u)[lane];
            return v10;
        }
        case 8:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r40 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r41 = bitcast<float>(v7.x);
            R.r42 = bitcast<float>(v7.y);
            R.r43 = bitcast<float>(v7.z);
            R.r44 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r45 = bitcast<float>(v8.x);
            R.r46 = bitcast<float>(v8.y);
            R.r47 = bitcast<float>(v8.z);
            R.r48 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r53 = bitcast<unsigned int>(v9.x);
            return v9.y;
        }
        case 9:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r40 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r41 = bitcast<float>(v7.x);
            R.r42 = bitcast<float>(v7.y);
            return v7.z;
        }
        case 10:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r49 = bitcast<unsigned int>(v5.x);
            R.r53 = bitcast<unsigned int>(v5.y);
            return v5.z;
        }
        case 11:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const unsigned v5 = reinterpret_cast<const unsigned*>(stage + 2560u)[lane];
            return v5;
        }
        case 12:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r28 = bitcast<float>(v4.y);
            R.r29 = bitcast<float>(v4.z);
            R.r30 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r31 = bitcast<float>(v5.x);
            R.r32 = bitcast<unsigned int>(v5.y);
            R.r33 = bitcast<unsigned int>(v5.z);
            R.r34 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r35 = bitcast<unsigned int>(v6.x);
            R.r36 = bitcast<float>(v6.y);
            R.r37 = bitcast<float>(v6.z);
            R.r38 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r39 = bitcast<float>(v7.x);
            R.r40 = bitcast<float>(v7.y);
            R.r41 = bitcast<float>(v7.z);
            R.r42 = bitcast<float>(v7.w);
            const uint2 v8 = reinterpret_cast<const uint2*>(stage + 4096u)[lane];
            R.r53 = bitcast<unsigned int>(v8.x);
            return v8.y;
        }
        case 13:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r53 = bitcast<unsigned int>(v7.z);
            return v7.w;
        }
        case 14:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r37 = bitcast<float>(v5.x);
            R.r38 = bitcast<float>(v5.y);
            R.r39 = bitcast<float>(v5.z);
            R.r40 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r41 = bitcast<float>(v6.x);
            R.r42 = bitcast<float>(v6.y);
            R.r53 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 15:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r49 = bitcast<unsigned int>(v5.x);
            R.r53 = bitcast<unsigned int>(v5.y);
            return v5.z;
        }
        case 16:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<unsigned int>(v4.w);
            const unsigned v5 = reinterpret_cast<const unsigned*>(stage + 2560u)[lane];
            return v5;
        }
        case 17:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r34 = bitcast<float>(v5.y);
            R.r35 = bitcast<unsigned int>(v5.z);
            R.r36 = bitcast<float>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(stage + 3072u)[lane];
            R.r53 = bitcast<unsigned int>(v6.x);
            return v6.y;
        }
        case 18:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r35 = bitcast<unsigned int>(v5.y);
            R.r36 = bitcast<float>(v5.z);
            R.r53 = bitcast<unsigned int>(v5.w);
            const unsigned v6 = reinterpret_cast<const unsigned*>(stage + 3072u)[lane];
            return v6;
        }
        case 19:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r35 = bitcast<unsigned int>(v5.y);
            R.r36 = bitcast<float>(v5.z);
            R.r49 = bitcast<unsigned int>(v5.w);
            const unsigned v6 = reinterpret_cast<const unsigned*>(stage + 3072u)[lane];
            return v6;
        }
        case 20:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r34 = bitcast<float>(v5.y);
            R.r35 = bitcast<unsigned int>(v5.z);
            R.r36 = bitcast<float>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(stage + 3072u)[lane];
            R.r53 = bitcast<unsigned int>(v6.x);
            return v6.y;
        }
        case 21:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r29 = bitcast<float>(v4.z);
            R.r31 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r32 = bitcast<unsigned int>(v5.x);
            R.r33 = bitcast<unsigned int>(v5.y);
            R.r34 = bitcast<float>(v5.z);
            R.r35 = bitcast<unsigned int>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(stage + 3072u)[lane];
            R.r36 = bitcast<float>(v6.x);
            return v6.y;
        }
        case 22:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r29 = bitcast<float>(v4.z);
            R.r31 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r32 = bitcast<unsigned int>(v5.x);
            R.r33 = bitcast<unsigned int>(v5.y);
            R.r36 = bitcast<float>(v5.z);
            R.r53 = bitcast<unsigned int>(v5.w);
            const unsigned v6 = reinterpret_cast<const unsigned*>(stage + 3072u)[lane];
            return v6;
        }
        case 23:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r29 = bitcast<float>(v4.z);
            R.r31 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r32 = bitcast<unsigned int>(v5.x);
            R.r33 = bitcast<unsigned int>(v5.y);
            R.r53 = bitcast<unsigned int>(v5.z);
            return v5.w;
        }
        case 24:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r49 = bitcast<unsigned int>(v5.y);
            R.r53 = bitcast<unsigned int>(v5.z);
            return v5.w;
        }
        case 25:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r49 = bitcast<unsigned int>(v5.x);
            R.r53 = bitcast<unsigned int>(v5.y);
            return v5.z;
        }
        case 26:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<unsigned int>(v4.w);
            const unsigned v5 = reinterpret_cast<const unsigned*>(stage + 2560u)[lane];
            return v5;
        }
        case 27:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r29 = bitcast<float>(v4.y);
            R.r31 = bitcast<float>(v4.z);
            R.r32 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r33 = bitcast<unsigned int>(v5.x);
            R.r49 = bitcast<unsigned int>(v5.y);
            R.r53 = bitcast<unsigned int>(v5.z);
            return v5.w;
        }
        case 28:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r34 = bitcast<float>(v6.x);
            R.r35 = bitcast<unsigned int>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 29:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r17 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<float>(v3.z);
            R.r21 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r27 = bitcast<float>(v4.y);
            R.r28 = bitcast<float>(v4.z);
            R.r29 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r30 = bitcast<float>(v5.x);
            R.r31 = bitcast<float>(v5.y);
            R.r32 = bitcast<unsigned int>(v5.z);
            R.r33 = bitcast<unsigned int>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(stage + 3072u)[lane];
            R.r53 = bitcast<unsigned int>(v6.x);
            return v6.y;
        }
        case 30:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r17 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<float>(v3.y);
            R.r21 = bitcast<float>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r27 = bitcast<float>(v4.x);
            R.r31 = bitcast<float>(v4.y);
            R.r32 = bitcast<unsigned int>(v4.z);
            R.r33 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r49 = bitcast<unsigned int>(v5.x);
            R.r53 = bitcast<unsigned int>(v5.y);
            return v5.z;
        }
        case 31:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r8 = bitcast<unsigned int>(v1.y);
            R.r9 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r17 = bitcast<unsigned int>(v2.z);
            R.r32 = bitcast<unsigned int>(v2.w);
            const uint2 v3 = reinterpret_cast<const uint2*>(stage + 1536u)[lane];
            R.r53 = bitcast<unsigned int>(v3.x);
            return v3.y;
        }
        case 32:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint2 v1 = reinterpret_cast<const uint2*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            return v1.y;
        }
        default: return 0xffffffffu;
        }
    }
};

const int kInTypes[] = {LOOM_B200_U32};
const int kOutTypes[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kInNames[] = {"ppp"};
const char* const kOutNames[] = {"L0", "L1", "L2", "rc", "ppp"};
const uint32_t kInstrs[] = {25, 335, 31, 11, 20, 3, 19, 10, 13, 22, 7, 28, 12, 15, 7, 7, 25, 3, 3, 3, 5, 11, 4, 3, 2, 4, 13, 15, 14, 16, 13, 20, 4};
const uint32_t kLive[] = {8, 48, 84, 148, 140, 140, 132, 160, 148, 120, 88, 80, 132, 124, 108, 88, 80, 100, 96, 96, 100, 100, 96, 92, 92, 88, 80, 92, 108, 100, 88, 52, 20};

const loom_b200_kernel_info kInfo = {
    "primary_const_b20_256", "1f441c05ae8a8bdc", 1u, 5u, kInTypes, kOutTypes, kInNames, kOutNames,
    33u, 54u, 216u, 46u, kInstrs, kLive};

const uint32_t kQRegs0[] = {1u, 53u};
const int kQTypes0[] = {LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames0[] = {"ppp", "ct"};
const unsigned long long kQOffs0[] = {0ull, 0ull};
const unsigned kQSubs0[] = {0u, 4u};
const unsigned kQWidths0[] = {16u, 16u};
const uint32_t kQRegs1[] = {1u, 2u, 3u, 4u, 5u, 8u, 9u, 12u, 13u, 15u, 17u, 53u};
const int kQTypes1[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames1[] = {"ppp", "L0", "L1", "L2", "rc", "c0", "c1", "pp0", "pp1", "pw", "sc", "ct"};
const unsigned long long kQOffs1[] = {16ull, 16ull, 16ull, 16ull, 32ull, 32ull, 32ull, 32ull, 48ull, 48ull, 48ull, 48ull};
const unsigned kQSubs1[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths1[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs2[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 53u};
const int kQTypes2[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames2[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "ct"};
const unsigned long long kQOffs2[] = {72ull, 72ull, 72ull, 72ull, 88ull, 88ull, 88ull, 88ull, 104ull, 104ull, 104ull, 104ull, 120ull, 120ull, 120ull, 120ull, 136ull, 136ull, 136ull, 136ull, 152ull};
const unsigned kQSubs2[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths2[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs3[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 50u, 51u, 52u, 53u};
const int kQTypes3[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames3[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "vr60", "vr61", "vr62", "ct"};
const unsigned long long kQOffs3[] = {160ull, 160ull, 160ull, 160ull, 176ull, 176ull, 176ull, 176ull, 192ull, 192ull, 192ull, 192ull, 208ull, 208ull, 208ull, 208ull, 224ull, 224ull, 224ull, 224ull, 240ull, 240ull, 240ull, 240ull, 256ull, 256ull, 256ull, 256ull, 272ull, 272ull, 272ull, 272ull, 288ull, 288ull, 288ull, 288ull, 304ull};
const unsigned kQSubs3[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths3[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs4[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 10u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 53u};
const int kQTypes4[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames4[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "tmp1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct"};
const unsigned long long kQOffs4[] = {312ull, 312ull, 312ull, 312ull, 328ull, 328ull, 328ull, 328ull, 344ull, 344ull, 344ull, 344ull, 360ull, 360ull, 360ull, 360ull, 376ull, 376ull, 376ull, 376ull, 392ull, 392ull, 392ull, 392ull, 408ull, 408ull, 408ull, 408ull, 424ull, 424ull, 424ull, 424ull, 440ull, 440ull, 440ull};
const unsigned kQSubs4[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths4[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs5[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 10u, 11u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u};
const int kQTypes5[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames5[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "tmp1", "tmp2", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32"};
const unsigned long long kQOffs5[] = {456ull, 456ull, 456ull, 456ull, 472ull, 472ull, 472ull, 472ull, 488ull, 488ull, 488ull, 488ull, 504ull, 504ull, 504ull, 504ull, 520ull, 520ull, 520ull, 520ull, 536ull, 536ull, 536ull, 536ull, 552ull, 552ull, 552ull, 552ull, 568ull, 568ull, 568ull, 568ull, 584ull, 584ull, 584ull};
const unsigned kQSubs5[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths5[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs6[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u};
const int kQTypes6[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames6[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32"};
const unsigned long long kQOffs6[] = {600ull, 600ull, 600ull, 600ull, 616ull, 616ull, 616ull, 616ull, 632ull, 632ull, 632ull, 632ull, 648ull, 648ull, 648ull, 648ull, 664ull, 664ull, 664ull, 664ull, 680ull, 680ull, 680ull, 680ull, 696ull, 696ull, 696ull, 696ull, 712ull, 712ull, 712ull, 712ull, 728ull};
const unsigned kQSubs6[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths6[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs7[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 50u, 51u, 52u, 53u};
const int kQTypes7[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames7[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "vr40", "vr41", "vr42", "vr60", "vr61", "vr62", "ct"};
const unsigned long long kQOffs7[] = {736ull, 736ull, 736ull, 736ull, 752ull, 752ull, 752ull, 752ull, 768ull, 768ull, 768ull, 768ull, 784ull, 784ull, 784ull, 784ull, 800ull, 800ull, 800ull, 800ull, 816ull, 816ull, 816ull, 816ull, 832ull, 832ull, 832ull, 832ull, 848ull, 848ull, 848ull, 848ull, 864ull, 864ull, 864ull, 864ull, 880ull, 880ull, 880ull, 880ull};
const unsigned kQSubs7[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths7[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs8[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 48u, 53u};
const int kQTypes8[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames8[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr30", "vr31", "vr32", "vr40", "vr41", "vr42", "vr50", "vr51", "vr52", "ct"};
const unsigned long long kQOffs8[] = {904ull, 904ull, 904ull, 904ull, 920ull, 920ull, 920ull, 920ull, 936ull, 936ull, 936ull, 936ull, 952ull, 952ull, 952ull, 952ull, 968ull, 968ull, 968ull, 968ull, 984ull, 984ull, 984ull, 984ull, 1000ull, 1000ull, 1000ull, 1000ull, 1016ull, 1016ull, 1016ull, 1016ull, 1032ull, 1032ull, 1032ull, 1032ull, 1048ull};
const unsigned kQSubs8[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths8[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs9[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 40u, 41u, 42u};
const int kQTypes9[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames9[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr30", "vr31", "vr32"};
const unsigned long long kQOffs9[] = {1056ull, 1056ull, 1056ull, 1056ull, 1072ull, 1072ull, 1072ull, 1072ull, 1088ull, 1088ull, 1088ull, 1088ull, 1104ull, 1104ull, 1104ull, 1104ull, 1120ull, 1120ull, 1120ull, 1120ull, 1136ull, 1136ull, 1136ull, 1136ull, 1152ull, 1152ull, 1152ull, 1152ull, 1168ull, 1168ull};
const unsigned kQSubs9[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths9[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs10[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes10[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames10[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs10[] = {1184ull, 1184ull, 1184ull, 1184ull, 1200ull, 1200ull, 1200ull, 1200ull, 1216ull, 1216ull, 1216ull, 1216ull, 1232ull, 1232ull, 1232ull, 1232ull, 1248ull, 1248ull, 1248ull, 1248ull, 1264ull, 1264ull};
const unsigned kQSubs10[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths10[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs11[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u};
const int kQTypes11[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames11[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp"};
const unsigned long long kQOffs11[] = {1280ull, 1280ull, 1280ull, 1280ull, 1296ull, 1296ull, 1296ull, 1296ull, 1312ull, 1312ull, 1312ull, 1312ull, 1328ull, 1328ull, 1328ull, 1328ull, 1344ull, 1344ull, 1344ull, 1344ull};
const unsigned kQSubs11[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths11[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs12[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 53u};
const int kQTypes12[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames12[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct"};
const unsigned long long kQOffs12[] = {1368ull, 1368ull, 1368ull, 1368ull, 1384ull, 1384ull, 1384ull, 1384ull, 1400ull, 1400ull, 1400ull, 1400ull, 1416ull, 1416ull, 1416ull, 1416ull, 1432ull, 1432ull, 1432ull, 1432ull, 1448ull, 1448ull, 1448ull, 1448ull, 1464ull, 1464ull, 1464ull, 1464ull, 1480ull, 1480ull, 1480ull, 1480ull, 1496ull};
const unsigned kQSubs12[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths12[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs13[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 53u};
const int kQTypes13[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames13[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "ct"};
const unsigned long long kQOffs13[] = {1504ull, 1504ull, 1504ull, 1504ull, 1520ull, 1520ull, 1520ull, 1520ull, 1536ull, 1536ull, 1536ull, 1536ull, 1552ull, 1552ull, 1552ull, 1552ull, 1568ull, 1568ull, 1568ull, 1568ull, 1584ull, 1584ull, 1584ull, 1584ull, 1600ull, 1600ull, 1600ull, 1600ull, 1616ull, 1616ull, 1616ull};
const unsigned kQSubs13[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths13[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs14[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 37u, 38u, 39u, 40u, 41u, 42u, 53u};
const int kQTypes14[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames14[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct"};
const unsigned long long kQOffs14[] = {1632ull, 1632ull, 1632ull, 1632ull, 1648ull, 1648ull, 1648ull, 1648ull, 1664ull, 1664ull, 1664ull, 1664ull, 1680ull, 1680ull, 1680ull, 1680ull, 1696ull, 1696ull, 1696ull, 1696ull, 1712ull, 1712ull, 1712ull, 1712ull, 1728ull, 1728ull, 1728ull};
const unsigned kQSubs14[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths14[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs15[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes15[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames15[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs15[] = {1744ull, 1744ull, 1744ull, 1744ull, 1760ull, 1760ull, 1760ull, 1760ull, 1776ull, 1776ull, 1776ull, 1776ull, 1792ull, 1792ull, 1792ull, 1792ull, 1808ull, 1808ull, 1808ull, 1808ull, 1824ull, 1824ull};
const unsigned kQSubs15[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths15[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs16[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 53u};
const int kQTypes16[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames16[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "ct"};
const unsigned long long kQOffs16[] = {1840ull, 1840ull, 1840ull, 1840ull, 1856ull, 1856ull, 1856ull, 1856ull, 1872ull, 1872ull, 1872ull, 1872ull, 1888ull, 1888ull, 1888ull, 1888ull, 1904ull, 1904ull, 1904ull, 1904ull};
const unsigned kQSubs16[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths16[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs17[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 34u, 35u, 36u, 53u};
const int kQTypes17[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames17[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "ct"};
const unsigned long long kQOffs17[] = {1928ull, 1928ull, 1928ull, 1928ull, 1944ull, 1944ull, 1944ull, 1944ull, 1960ull, 1960ull, 1960ull, 1960ull, 1976ull, 1976ull, 1976ull, 1976ull, 1992ull, 1992ull, 1992ull, 1992ull, 2008ull, 2008ull, 2008ull, 2008ull, 2024ull};
const unsigned kQSubs17[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths17[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs18[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 35u, 36u, 53u};
const int kQTypes18[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames18[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr11", "vr12", "ct"};
const unsigned long long kQOffs18[] = {2032ull, 2032ull, 2032ull, 2032ull, 2048ull, 2048ull, 2048ull, 2048ull, 2064ull, 2064ull, 2064ull, 2064ull, 2080ull, 2080ull, 2080ull, 2080ull, 2096ull, 2096ull, 2096ull, 2096ull, 2112ull, 2112ull, 2112ull, 2112ull};
const unsigned kQSubs18[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths18[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs19[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 35u, 36u, 49u};
const int kQTypes19[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames19[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr11", "vr12", "hit"};
const unsigned long long kQOffs19[] = {2136ull, 2136ull, 2136ull, 2136ull, 2152ull, 2152ull, 2152ull, 2152ull, 2168ull, 2168ull, 2168ull, 2168ull, 2184ull, 2184ull, 2184ull, 2184ull, 2200ull, 2200ull, 2200ull, 2200ull, 2216ull, 2216ull, 2216ull, 2216ull};
const unsigned kQSubs19[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths19[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs20[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 34u, 35u, 36u, 53u};
const int kQTypes20[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames20[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "ct"};
const unsigned long long kQOffs20[] = {2240ull, 2240ull, 2240ull, 2240ull, 2256ull, 2256ull, 2256ull, 2256ull, 2272ull, 2272ull, 2272ull, 2272ull, 2288ull, 2288ull, 2288ull, 2288ull, 2304ull, 2304ull, 2304ull, 2304ull, 2320ull, 2320ull, 2320ull, 2320ull, 2336ull};
const unsigned kQSubs20[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths20[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs21[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 34u, 35u, 36u};
const int kQTypes21[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32};
const char* const kQNames21[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12"};
const unsigned long long kQOffs21[] = {2344ull, 2344ull, 2344ull, 2344ull, 2360ull, 2360ull, 2360ull, 2360ull, 2376ull, 2376ull, 2376ull, 2376ull, 2392ull, 2392ull, 2392ull, 2392ull, 2408ull, 2408ull, 2408ull, 2408ull, 2424ull, 2424ull, 2424ull, 2424ull, 2440ull};
const unsigned kQSubs21[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths21[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs22[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 36u, 53u};
const int kQTypes22[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames22[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr12", "ct"};
const unsigned long long kQOffs22[] = {2448ull, 2448ull, 2448ull, 2448ull, 2464ull, 2464ull, 2464ull, 2464ull, 2480ull, 2480ull, 2480ull, 2480ull, 2496ull, 2496ull, 2496ull, 2496ull, 2512ull, 2512ull, 2512ull, 2512ull, 2528ull, 2528ull, 2528ull, 2528ull};
const unsigned kQSubs22[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths22[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs23[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 53u};
const int kQTypes23[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames23[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "ct"};
const unsigned long long kQOffs23[] = {2552ull, 2552ull, 2552ull, 2552ull, 2568ull, 2568ull, 2568ull, 2568ull, 2584ull, 2584ull, 2584ull, 2584ull, 2600ull, 2600ull, 2600ull, 2600ull, 2616ull, 2616ull, 2616ull, 2616ull, 2632ull, 2632ull, 2632ull};
const unsigned kQSubs23[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths23[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs24[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes24[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames24[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs24[] = {2648ull, 2648ull, 2648ull, 2648ull, 2664ull, 2664ull, 2664ull, 2664ull, 2680ull, 2680ull, 2680ull, 2680ull, 2696ull, 2696ull, 2696ull, 2696ull, 2712ull, 2712ull, 2712ull, 2712ull, 2728ull, 2728ull, 2728ull};
const unsigned kQSubs24[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths24[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs25[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes25[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames25[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs25[] = {2744ull, 2744ull, 2744ull, 2744ull, 2760ull, 2760ull, 2760ull, 2760ull, 2776ull, 2776ull, 2776ull, 2776ull, 2792ull, 2792ull, 2792ull, 2792ull, 2808ull, 2808ull, 2808ull, 2808ull, 2824ull, 2824ull};
const unsigned kQSubs25[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths25[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs26[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 53u};
const int kQTypes26[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames26[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "ct"};
const unsigned long long kQOffs26[] = {2840ull, 2840ull, 2840ull, 2840ull, 2856ull, 2856ull, 2856ull, 2856ull, 2872ull, 2872ull, 2872ull, 2872ull, 2888ull, 2888ull, 2888ull, 2888ull, 2904ull, 2904ull, 2904ull, 2904ull};
const unsigned kQSubs26[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths26[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs27[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes27[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames27[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs27[] = {2928ull, 2928ull, 2928ull, 2928ull, 2944ull, 2944ull, 2944ull, 2944ull, 2960ull, 2960ull, 2960ull, 2960ull, 2976ull, 2976ull, 2976ull, 2976ull, 2992ull, 2992ull, 2992ull, 2992ull, 3008ull, 3008ull, 3008ull};
const unsigned kQSubs27[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths27[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs28[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u};
const int kQTypes28[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32};
const char* const kQNames28[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12"};
const unsigned long long kQOffs28[] = {3024ull, 3024ull, 3024ull, 3024ull, 3040ull, 3040ull, 3040ull, 3040ull, 3056ull, 3056ull, 3056ull, 3056ull, 3072ull, 3072ull, 3072ull, 3072ull, 3088ull, 3088ull, 3088ull, 3088ull, 3104ull, 3104ull, 3104ull, 3104ull, 3120ull, 3120ull, 3120ull};
const unsigned kQSubs28[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths28[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs29[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 53u};
const int kQTypes29[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames29[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "ct"};
const unsigned long long kQOffs29[] = {3136ull, 3136ull, 3136ull, 3136ull, 3152ull, 3152ull, 3152ull, 3152ull, 3168ull, 3168ull, 3168ull, 3168ull, 3184ull, 3184ull, 3184ull, 3184ull, 3200ull, 3200ull, 3200ull, 3200ull, 3216ull, 3216ull, 3216ull, 3216ull, 3232ull};
const unsigned kQSubs29[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths29[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs30[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes30[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames30[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs30[] = {3240ull, 3240ull, 3240ull, 3240ull, 3256ull, 3256ull, 3256ull, 3256ull, 3272ull, 3272ull, 3272ull, 3272ull, 3288ull, 3288ull, 3288ull, 3288ull, 3304ull, 3304ull, 3304ull, 3304ull, 3320ull, 3320ull};
const unsigned kQSubs30[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths30[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs31[] = {1u, 2u, 3u, 4u, 5u, 8u, 9u, 12u, 13u, 15u, 17u, 32u, 53u};
const int kQTypes31[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames31[] = {"ppp", "L0", "L1", "L2", "rc", "c0", "c1", "pp0", "pp1", "pw", "sc", "pid", "ct"};
const unsigned long long kQOffs31[] = {3336ull, 3336ull, 3336ull, 3336ull, 3352ull, 3352ull, 3352ull, 3352ull, 3368ull, 3368ull, 3368ull, 3368ull, 3384ull};
const unsigned kQSubs31[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths31[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs32[] = {1u, 2u, 3u, 4u, 5u};
const int kQTypes32[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames32[] = {"ppp", "L0", "L1", "L2", "rc"};
const unsigned long long kQOffs32[] = {3392ull, 3392ull, 3392ull, 3392ull, 3408ull};
const unsigned kQSubs32[] = {0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths32[] = {16u, 16u, 16u, 16u, 8u};
const loom_b200_queue_layout kQueues[] = {
    {0u, -1, 2u, kQRegs0, kQTypes0, kQNames0},
    {1u, -1, 12u, kQRegs1, kQTypes1, kQNames1},
    {2u, -1, 21u, kQRegs2, kQTypes2, kQNames2},
    {3u, -1, 37u, kQRegs3, kQTypes3, kQNames3},
    {4u, -1, 35u, kQRegs4, kQTypes4, kQNames4},
    {5u, -1, 35u, kQRegs5, kQTypes5, kQNames5},
    {6u, -1, 33u, kQRegs6, kQTypes6, kQNames6},
    {7u, -1, 40u, kQRegs7, kQTypes7, kQNames7},
    {8u, -1, 37u, kQRegs8, kQTypes8, kQNames8},
    {9u, -1, 30u, kQRegs9, kQTypes9, kQNames9},
    {10u, -1, 22u, kQRegs10, kQTypes10, kQNames10},
    {11u, -1, 20u, kQRegs11, kQTypes11, kQNames11},
    {12u, -1, 33u, kQRegs12, kQTypes12, kQNames12},
    {13u, -1, 31u, kQRegs13, kQTypes13, kQNames13},
    {14u, -1, 27u, kQRegs14, kQTypes14, kQNames14},
    {15u, -1, 22u, kQRegs15, kQTypes15, kQNames15},
    {16u, -1, 20u, kQRegs16, kQTypes16, kQNames16},
    {17u, -1, 25u, kQRegs17, kQTypes17, kQNames17},
    {18u, -1, 24u, kQRegs18, kQTypes18, kQNames18},
    {19u, -1, 24u, kQRegs19, kQTypes19, kQNames19},
    {20u, -1, 25u, kQRegs20, kQTypes20, kQNames20},
    {21u, -1, 25u, kQRegs21, kQTypes21, kQNames21},
    {22u, -1, 24u, kQRegs22, kQTypes22, kQNames22},
    {23u, -1, 23u, kQRegs23, kQTypes23, kQNames23},
    {24u, -1, 23u, kQRegs24, kQTypes24, kQNames24},
    {25u, -1, 22u, kQRegs25, kQTypes25, kQNames25},
    {26u, -1, 20u, kQRegs26, kQTypes26, kQNames26},
    {27u, -1, 23u, kQRegs27, kQTypes27, kQNames27},
    {28u, -1, 27u, kQRegs28, kQTypes28, kQNames28},
    {29u, -1, 25u, kQRegs29, kQTypes29, kQNames29},
    {30u, -1, 22u, kQRegs30, kQTypes30, kQNames30},
    {31u, -1, 13u, kQRegs31, kQTypes31, kQNames31},
    {32u, -1, 5u, kQRegs32, kQTypes32, kQNames32},
};
const QueueSegment kSegments[] = {
    {kQOffs0, kQSubs0, kQWidths0, 0ull, 8u, 16u},
    {kQOffs1, kQSubs1, kQWidths1, 64ull, 0u, 4u},
    {kQOffs2, kQSubs2, kQWidths2, 152ull, 4u, 8u},
    {kQOffs3, kQSubs3, kQWidths3, 304ull, 4u, 8u},
    {kQOffs4, kQSubs4, kQWidths4, 440ull, 12u, 16u},
    {kQOffs5, kQSubs5, kQWidths5, 584ull, 12u, 16u},
    {kQOffs6, kQSubs6, kQWidths6, 728ull, 4u, 8u},
    {kQOffs7, kQSubs7, kQWidths7, 896ull, 0u, 4u},
    {kQOffs8, kQSubs8, kQWidths8, 1048ull, 4u, 8u},
    {kQOffs9, kQSubs9, kQWidths9, 1168ull, 8u, 16u},
    {kQOffs10, kQSubs10, kQWidths10, 1264ull, 8u, 16u},
    {kQOffs11, kQSubs11, kQWidths11, 1360ull, 0u, 4u},
    {kQOffs12, kQSubs12, kQWidths12, 1496ull, 4u, 8u},
    {kQOffs13, kQSubs13, kQWidths13, 1616ull, 12u, 16u},
    {kQOffs14, kQSubs14, kQWidths14, 1728ull, 12u, 16u},
    {kQOffs15, kQSubs15, kQWidths15, 1824ull, 8u, 16u},
    {kQOffs16, kQSubs16, kQWidths16, 1920ull, 0u, 4u},
    {kQOffs17, kQSubs17, kQWidths17, 2024ull, 4u, 8u},
    {kQOffs18, kQSubs18, kQWidths18, 2128ull, 0u, 4u},
    {kQOffs19, kQSubs19, kQWidths19, 2232ull, 0u, 4u},
    {kQOffs20, kQSubs20, kQWidths20, 2336ull, 4u, 8u},
    {kQOffs21, kQSubs21, kQWidths21, 2440ull, 4u, 8u},
    {kQOffs22, kQSubs22, kQWidths22, 2544ull, 0u, 4u},
    {kQOffs23, kQSubs23, kQWidths23, 2632ull, 12u, 16u},
    {kQOffs24, kQSubs24, kQWidths24, 2728ull, 12u, 16u},
    {kQOffs25, kQSubs25, kQWidths25, 2824ull, 8u, 16u},
    {kQOffs26, kQSubs26, kQWidths26, 2920ull, 0u, 4u},
    {kQOffs27, kQSubs27, kQWidths27, 3008ull, 12u, 16u},
    {kQOffs28, kQSubs28, kQWidths28, 3120ull, 12u, 16u},
    {kQOffs29, kQSubs29, kQWidths29, 3232ull, 4u, 8u},
    {kQOffs30, kQSubs30, kQWidths30, 3320ull, 8u, 16u},
    {kQOffs31, kQSubs31, kQWidths31, 3384ull, 4u, 8u},
    {kQOffs32, kQSubs32, kQWidths32, 3408ull, 4u, 8u},
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

const unsigned kRegCaps[] = {64u, 32u, 40u, 48u, 56u, 80u, 96u, 128u};

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
    case 32u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 32, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 32, false, false>);
    case 40u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 40, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 40, false, false>);
    case 48u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 48, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 48, false, false>);
    case 56u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 56, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 56, false, false>);
    case 80u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 80, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 80, false, false>);
    case 96u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 96, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 96, false, false>);
    case 128u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, 128, false, true>)
                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, 128, false, false>);
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

} } // namespace loom_b200::k_primary_const_b20_256

extern const loom_b200::KernelEntry loom_b200_entry_primary_const_b20_256;
const loom_b200::KernelEntry loom_b200_entry_primary_const_b20_256 = {
    &loom_b200::k_primary_const_b20_256::kInfo, loom_b200::k_primary_const_b20_256::K::kRowBytes, 33,
    &loom_b200::k_primary_const_b20_256::launch_plain, &loom_b200::k_primary_const_b20_256::launch_regroup,
    &loom_b200::k_primary_const_b20_256::regroup_occupancy,
    loom_b200::k_primary_const_b20_256::kQueues, loom_b200::k_primary_const_b20_256::kSegments,
    loom_b200::k_primary_const_b20_256::kRegCaps, 8u, loom_b200::k_primary_const_b20_256::K::kMaxStageRow};
