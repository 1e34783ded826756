// Generated by loom_b200.codegen from loom_b200/ir/pt_const_40.lir.
// Kernel IR digest 107b56955f2949d4; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_pt_const_40 {

__constant__ unsigned kInstrTab[44] = {27, 296, 34, 10, 31, 11, 20, 3, 19, 10, 13, 22, 7, 28, 12, 15, 7, 7, 25, 3, 3, 3, 5, 11, 4, 3, 2, 4, 13, 15, 14, 16, 13, 2, 10, 31, 4, 19, 12, 12, 2, 70, 23, 5};
__constant__ unsigned kLiveTab[44] = {64, 124, 76, 120, 132, 196, 188, 188, 180, 208, 196, 168, 136, 128, 180, 172, 156, 136, 128, 148, 144, 144, 148, 148, 144, 140, 140, 136, 128, 140, 156, 148, 136, 128, 128, 104, 112, 124, 108, 108, 120, 116, 120, 24};
__constant__ int kQueueBlock[44] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43};
__constant__ unsigned kQuorumTab[44] = {8, 26, 9, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 3, 0, 0, 0, 0, 0, 13, 0, 0};
__constant__ unsigned kRankTab[44] = {0, 1, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 25, 26, 21, 22, 23, 24, 27, 28, 29, 30, 31, 32, 33, 34, 35, 38, 42, 41, 40, 39, 43, 2, 36, 37};

struct K
{
    static constexpr int kNumBlocks = 44;
    static constexpr int kNumQueues = 44;
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
        float r16; // mean: f32
        float r17; // m2: f32
        unsigned int r18; // rpt: u32
        unsigned int r19; // ns: f32,u32
        unsigned int r20; // u0: f32,u32
        unsigned int r21; // u1: f32,u32
        float r22; // o0: f32
        float r23; // o1: f32
        float r24; // o2: f32
        float r25; // PL0: f32
        float r26; // PL1: f32
        float r27; // PL2: f32
        float r28; // clr0: f32
        float r29; // clr1: f32
        float r30; // clr2: f32
        unsigned int r31; // depth: u32
        float r32; // d2: f32
        float r33; // vr00: f32
        float r34; // vr01: f32
        float r35; // vr02: f32
        float r36; // t: f32
        unsigned int r37; // pid: u32
        unsigned int r38; // rp: u32
        float r39; // vr10: f32
        unsigned int r40; // vr11: u32,f32
        float r41; // vr12: f32
        float r42; // vr20: f32
        float r43; // vr21: f32
        float r44; // vr22: f32
        float r45; // vr30: f32
        float r46; // vr31: f32
        float r47; // vr32: f32
        float r48; // vr40: f32
        float r49; // vr41: f32
        float r50; // vr42: f32
        float r51; // vr50: f32
        float r52; // vr51: f32
        float r53; // vr52: f32
        unsigned int r54; // hit: u32,f32
        float r55; // vr60: f32
        float r56; // vr61: f32
        float r57; // vr62: f32
        unsigned int r58; // ct: u32,f32
        float r59; // t0: f32
        float r60; // t1: f32
        float r61; // t2: f32
        float r62; // n0: f32
        float r63; // n1: f32
        float r64; // n2: f32
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
        R.r22 = 0;
        R.r23 = 0;
        R.r24 = 0;
        R.r25 = 0;
        R.r26 = 0;
        R.r27 = 0;
        R.r28 = 0;
        R.r29 = 0;
        R.r30 = 0;
        R.r31 = 0;
        R.r32 = 0;
        R.r58 = 0;
        R.r62 = 0;
        R.r63 = 0;
        R.r64 = 0;
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
        case 33: goto L_B33;
        case 34: goto L_B34;
        case 35: goto L_B35;
        case 36: goto L_B36;
        case 37: goto L_B37;
        case 38: goto L_B38;
        case 39: goto L_B39;
        case 40: goto L_B40;
        case 41: goto L_B41;
        case 42: goto L_B42;
        case 43: goto L_B43;
        default: return kHalt;
        }
    L_B0: // START
        if(stop_heavy && !fresh) return 0;
    L_B0_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 0, 27u);
        R.r6 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r1) >> static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r7 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r1) & static_cast<unsigned int>(((unsigned int)0xffffull))));
        R.r8 = static_cast<unsigned int>(R.r6);
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) * static_cast<unsigned int>(((unsigned int)0x28ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) + static_cast<unsigned int>(R.r7)));
        R.r9 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x1.4000000000000p+5f)));
        R.r11 = bitcast<unsigned int>(static_cast<float>((0x1.4000000000000p+5f)));
        R.r12 = static_cast<float>(R.r6);
        R.r13 = static_cast<float>(R.r7);
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) / static_cast<float>(bitcast<float>(R.r11)))));
        R.r15 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) / static_cast<float>(bitcast<float>(R.r10))));
        R.r15 = static_cast<float>(static_cast<float>(static_cast<float>(R.r15) * static_cast<float>((0x1.0000000000000p+0f))));
        R.r16 = static_cast<float>((0x0.0p+0f));
        R.r17 = static_cast<float>((0x0.0p+0f));
        R.r12 = static_cast<float>(static_cast<float>(static_cast<float>(R.r12) / static_cast<float>(bitcast<float>(R.r10))));
        R.r12 = static_cast<float>(static_cast<float>(static_cast<float>(R.r12) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r12 = static_cast<float>(static_cast<float>(static_cast<float>(R.r12) * static_cast<float>(bitcast<float>(R.r14))));
        R.r13 = static_cast<float>(static_cast<float>(static_cast<float>(R.r13) / static_cast<float>(bitcast<float>(R.r11))));
        R.r13 = static_cast<float>(static_cast<float>(static_cast<float>(R.r13) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r2 = static_cast<float>((0x0.0p+0f));
        R.r3 = static_cast<float>((0x0.0p+0f));
        R.r4 = static_cast<float>((0x0.0p+0f));
        R.r5 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r19 = static_cast<unsigned int>(((unsigned int)0x0ull));
        goto L_B1;
    L_B1: // roll
        if(stop_heavy && !fresh) return 1;
    L_B1_again:
        if(budget == 0u) return 1;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 1, 296u);
        R.r20 = static_cast<unsigned int>(R.r8);
        R.r21 = static_cast<unsigned int>(R.r9);
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x3ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x7ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r10)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r10)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) + static_cast<unsigned int>(((unsigned int)0x2611501ull))));
        R.r10 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r14) < static_cast<unsigned int>(R.r8)));
        R.r11 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r9) + static_cast<unsigned int>(R.r14)));
        R.r9 = static_cast<unsigned int>(((R.r10) ? (R.r11) : (R.r9)));
        R.r8 = static_cast<unsigned int>(((R.r10) ? (((unsigned int)0x0ull)) : (R.r14)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) >> static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) | static_cast<unsigned int>(((unsigned int)0x3f800000ull))));
        R.r20 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) - static_cast<float>((0x1.0000000000000p+0f)))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) | static_cast<unsigned int>(((unsigned int)0x3f800000ull))));
        R.r21 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r21)) - static_cast<float>((0x1.0000000000000p+0f)))));
        switch(R.r18) {
        case 0: goto L_B2;
        case 1: goto L_B3;
        case 2: goto L_B41;
        default: goto L_HALT;
        }
    L_B2: // sample_pixel
        if(stop_heavy && !fresh) return 2;
    L_B2_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 2, 34u);
        R.r22 = static_cast<float>((0x0.0p+0f));
        R.r23 = static_cast<float>((0x0.0p+0f));
        R.r24 = static_cast<float>((0x1.0000000000000p+1f));
        R.r25 = static_cast<float>((0x1.0000000000000p+0f));
        R.r26 = static_cast<float>((0x1.0000000000000p+0f));
        R.r27 = static_cast<float>((0x1.0000000000000p+0f));
        R.r6 = bitcast<unsigned int>(static_cast<float>(R.r12));
        R.r7 = bitcast<unsigned int>(static_cast<float>(R.r13));
        R.r28 = static_cast<float>((0x0.0p+0f));
        R.r29 = static_cast<float>((0x0.0p+0f));
        R.r30 = static_cast<float>((0x0.0p+0f));
        R.r31 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r15) * static_cast<float>((0x1.0000000000000p-1f)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) - static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) - static_cast<float>(bitcast<float>(R.r14)))));
        R.r20 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) * static_cast<float>(R.r15))));
        R.r21 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r21)) * static_cast<float>(R.r15))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) + static_cast<float>(bitcast<float>(R.r20)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) + static_cast<float>(bitcast<float>(R.r21)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>((0x1.6d9b200000000p+0f)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>((0x1.6d9b200000000p+0f)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r6)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r7)))));
        R.r32 = static_cast<float>((-0x1.0000000000000p+0f));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r32, R.r32, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r32 = static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(bitcast<float>(R.r14))));
        goto L_B3;
    L_B3: // traverse_scene
        fresh = false;
        if constexpr(kProf) count_block(ctx, 3, 10u);
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>((0x1.0624de0000000p-10f))));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>((0x1.0624de0000000p-10f))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>((0x1.0624de0000000p-10f))));
        R.r22 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) + static_cast<float>(R.r33)));
        R.r23 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) + static_cast<float>(R.r34)));
        R.r24 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) + static_cast<float>(R.r35)));
        R.r36 = static_cast<float>((0x1.e848000000000p+19f));
        R.r37 = static_cast<unsigned int>(((unsigned int)0xcull));
        R.r38 = static_cast<unsigned int>(((unsigned int)0x0ull));
        goto L_B4;
    L_B4: // traverse_box
        if(budget == 0u) return 4;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 4, 31u);
        R.r33 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : ((R.r38) == 2 ? (0x1.0000000000000p+0f) : ((R.r38) == 3 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r34 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : ((R.r38) == 2 ? (-0x1.0000000000000p+0f) : ((R.r38) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r35 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (0x1.0000000000000p+0f) : ((R.r38) == 1 ? (0x1.0000000000000p+0f) : ((R.r38) == 2 ? (-0x1.0000000000000p+0f) : ((R.r38) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r39 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : ((R.r38) == 2 ? (0x1.0000000000000p+0f) : ((R.r38) == 3 ? (-0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r40 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : ((R.r38) == 2 ? (-0x1.0000000000000p+0f) : ((R.r38) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f))))))));
        R.r41 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : ((R.r38) == 2 ? (0x1.0000000000000p+0f) : ((R.r38) == 3 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r42 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : ((R.r38) == 2 ? (0x1.0000000000000p+0f) : ((R.r38) == 3 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r43 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (0x1.0000000000000p+0f) : ((R.r38) == 2 ? (0x1.0000000000000p+0f) : ((R.r38) == 3 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r44 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : ((R.r38) == 2 ? (0x1.0000000000000p+0f) : ((R.r38) == 3 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r45 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : ((R.r38) == 2 ? (0x1.0000000000000p+0f) : ((R.r38) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r46 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (0x1.0000000000000p+0f) : ((R.r38) == 2 ? (0x1.0000000000000p+0f) : ((R.r38) == 3 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r47 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (0x1.0000000000000p+0f) : ((R.r38) == 2 ? (-0x1.0000000000000p+0f) : ((R.r38) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r48 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) - static_cast<float>(R.r33)));
        R.r49 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>(R.r34)));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) - static_cast<float>(R.r35)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r39) - static_cast<float>(R.r33)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r40)) - static_cast<float>(R.r34)));
        R.r53 = static_cast<float>(static_cast<float>(static_cast<float>(R.r41) - static_cast<float>(R.r35)));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(R.r52))));
        R.r55 = static_cast<float>(op_fma(bitcast<float>(R.r7), R.r53, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r53))));
        R.r56 = static_cast<float>(op_fma(R.r32, R.r51, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r51))));
        R.r57 = static_cast<float>(op_fma(bitcast<float>(R.r6), R.r52, (-(bitcast<float>(R.r54)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r48, R.r55, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r49, R.r56, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r50, R.r57, bitcast<float>(R.r14))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r14)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r10)) >= static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r54) goto L_B5; else goto L_B12;
    L_B5: // isect_quad_l1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 5, 11u);
        R.r48 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r33)));
        R.r49 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r34)));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r35)));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r48, R.r55, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r49, R.r56, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r50, R.r57, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r10)) >= static_cast<float>((0x0.0p+0f))));
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r10)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r54) goto L_B6; else goto L_B12;
    L_B6: // isect_quad_l2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 6, 20u);
        R.r48 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) - static_cast<float>(R.r33)));
        R.r49 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>(R.r34)));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) - static_cast<float>(R.r35)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r33)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r34)));
        R.r53 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r35)));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r53) * static_cast<float>(R.r49))));
        R.r55 = static_cast<float>(op_fma(R.r52, R.r50, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r50))));
        R.r56 = static_cast<float>(op_fma(R.r53, R.r48, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r48))));
        R.r57 = static_cast<float>(op_fma(R.r51, R.r49, (-(bitcast<float>(R.r54)))));
        R.r11 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r11 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r55, bitcast<float>(R.r11))));
        R.r11 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r56, bitcast<float>(R.r11))));
        R.r11 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r32, R.r57, bitcast<float>(R.r11))));
        R.r11 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r11)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r11)) >= static_cast<float>((0x0.0p+0f))));
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r11)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r54) goto L_B7; else goto L_B12;
    L_B7: // isect_quad_l3
        fresh = false;
        if constexpr(kProf) count_block(ctx, 7, 3u);
        R.r58 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) + static_cast<float>(bitcast<float>(R.r11)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r58)) > static_cast<float>((0x1.0000000000000p+0f))));
        if(R.r54) goto L_B8; else goto L_B11;
    L_B8: // isect_quad_l4
        fresh = false;
        if constexpr(kProf) count_block(ctx, 8, 19u);
        R.r48 = static_cast<float>(static_cast<float>(static_cast<float>(R.r39) - static_cast<float>(R.r42)));
        R.r49 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r40)) - static_cast<float>(R.r43)));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r41) - static_cast<float>(R.r44)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) - static_cast<float>(R.r42)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>(R.r43)));
        R.r53 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) - static_cast<float>(R.r44)));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(R.r52))));
        R.r55 = static_cast<float>(op_fma(bitcast<float>(R.r7), R.r53, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r53))));
        R.r56 = static_cast<float>(op_fma(R.r32, R.r51, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r51))));
        R.r57 = static_cast<float>(op_fma(bitcast<float>(R.r6), R.r52, (-(bitcast<float>(R.r54)))));
        R.r58 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r48, R.r55, bitcast<float>(R.r58))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r49, R.r56, bitcast<float>(R.r58))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r50, R.r57, bitcast<float>(R.r58))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r58)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r54)) >= static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r54) goto L_B9; else goto L_B12;
    L_B9: // isect_quad_l5
        fresh = false;
        if constexpr(kProf) count_block(ctx, 9, 10u);
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r42)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r43)));
        R.r53 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r44)));
        R.r54 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r51, R.r55, bitcast<float>(R.r54))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r52, R.r56, bitcast<float>(R.r54))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r53, R.r57, bitcast<float>(R.r54))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r54)) / static_cast<float>(bitcast<float>(R.r58)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r54)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r54) goto L_B10; else goto L_B12;
    L_B10: // isect_quad_l6
        fresh = false;
        if constexpr(kProf) count_block(ctx, 10, 13u);
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r53) * static_cast<float>(R.r49))));
        R.r55 = static_cast<float>(op_fma(R.r52, R.r50, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r50))));
        R.r56 = static_cast<float>(op_fma(R.r53, R.r48, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r48))));
        R.r57 = static_cast<float>(op_fma(R.r51, R.r49, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r55, bitcast<float>(R.r54))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r56, bitcast<float>(R.r54))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r32, R.r57, bitcast<float>(R.r54))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r54)) / static_cast<float>(bitcast<float>(R.r58)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r54)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r54) goto L_B11; else goto L_B12;
    L_B11: // isect_quad_l7
        fresh = false;
        if constexpr(kProf) count_block(ctx, 11, 22u);
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) - static_cast<float>(R.r33)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>(R.r34)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) - static_cast<float>(R.r35)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r33)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r34)));
        R.r53 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r35)));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r53) * static_cast<float>(R.r46))));
        R.r55 = static_cast<float>(op_fma(R.r52, R.r47, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r47))));
        R.r56 = static_cast<float>(op_fma(R.r53, R.r45, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r45))));
        R.r57 = static_cast<float>(op_fma(R.r51, R.r46, (-(bitcast<float>(R.r54)))));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r39) - static_cast<float>(R.r33)));
        R.r40 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r40)) - static_cast<float>(R.r34))));
        R.r41 = static_cast<float>(static_cast<float>(static_cast<float>(R.r41) - static_cast<float>(R.r35)));
        R.r58 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r39, R.r55, bitcast<float>(R.r58))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r40), R.r56, bitcast<float>(R.r58))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r41, R.r57, bitcast<float>(R.r58))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r58)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r58)) >= static_cast<float>((0x0.0p+0f))));
        goto L_B12;
    L_B12: // isect_quad_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 12, 7u);
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r58)) < static_cast<float>(R.r36))));
        R.r36 = static_cast<float>(((R.r54) ? (bitcast<float>(R.r58)) : (R.r36)));
        R.r37 = static_cast<unsigned int>(((R.r54) ? (R.r38) : (R.r37)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r38) == static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r38 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r38) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r38 = static_cast<unsigned int>(((R.r14) ? (((unsigned int)0x0ull)) : (R.r38)));
        if(R.r14) goto L_B13; else goto L_B4;
    L_B13: // traverse_tetrahedron
        if(budget == 0u) return 13;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 13, 28u);
        R.r33 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.935f360000000p-1f) : ((R.r38) == 1 ? (-0x1.157b7e0000000p-1f) : (0x1.09d1420000000p-3f)))));
        R.r34 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))));
        R.r35 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.2cf8d20000000p-1f) : ((R.r38) == 1 ? (0x1.51b56e0000000p-2f) : (-0x1.5e2a2e0000000p-2f)))));
        R.r39 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.157b7e0000000p-1f) : ((R.r38) == 1 ? (0x1.09d1420000000p-3f) : (-0x1.935f360000000p-1f)))));
        R.r40 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r38) == 0 ? (-0x1.0000000000000p+0f) : ((R.r38) == 1 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f))))));
        R.r41 = static_cast<float>(static_cast<float>(((R.r38) == 0 ? (0x1.51b56e0000000p-2f) : ((R.r38) == 1 ? (-0x1.5e2a2e0000000p-2f) : (-0x1.2cf8d20000000p-1f)))));
        R.r42 = static_cast<float>((-0x1.9999980000000p-2f));
        R.r43 = static_cast<float>((-0x1.6b0f960000000p-3f));
        R.r44 = static_cast<float>((-0x1.9999980000000p-3f));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r39) - static_cast<float>(R.r33)));
        R.r40 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r40)) - static_cast<float>(R.r34))));
        R.r41 = static_cast<float>(static_cast<float>(static_cast<float>(R.r41) - static_cast<float>(R.r35)));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r33)));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r43) - static_cast<float>(R.r34)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r44) - static_cast<float>(R.r35)));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(R.r43))));
        R.r45 = static_cast<float>(op_fma(bitcast<float>(R.r7), R.r44, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r44))));
        R.r46 = static_cast<float>(op_fma(R.r32, R.r42, (-(bitcast<float>(R.r54)))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r42))));
        R.r47 = static_cast<float>(op_fma(bitcast<float>(R.r6), R.r43, (-(bitcast<float>(R.r54)))));
        R.r58 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r39, R.r45, bitcast<float>(R.r58))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r40), R.r46, bitcast<float>(R.r58))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r41, R.r47, bitcast<float>(R.r58))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r58)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r54) goto L_B14; else goto L_B17;
    L_B14: // isect_triangle_mid1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 14, 12u);
        R.r58 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(bitcast<float>(R.r58)))));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r33)));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r34)));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r35)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r33, R.r45, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r34, R.r46, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r47, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r58)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x0.0p+0f))));
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r54) goto L_B15; else goto L_B17;
    L_B15: // isect_triangle_mid2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 15, 15u);
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r40)))));
        R.r45 = static_cast<float>(op_fma(R.r34, R.r41, (-(bitcast<float>(R.r10)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r33) * static_cast<float>(R.r41))));
        R.r46 = static_cast<float>(op_fma(R.r35, R.r39, (-(bitcast<float>(R.r10)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r34) * static_cast<float>(R.r39))));
        R.r47 = static_cast<float>(op_fma(R.r33, bitcast<float>(R.r40), (-(bitcast<float>(R.r10)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r45, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r46, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r32, R.r47, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) * static_cast<float>(bitcast<float>(R.r58)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r10)) >= static_cast<float>((0x0.0p+0f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) + static_cast<float>(bitcast<float>(R.r10)))));
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r54) goto L_B16; else goto L_B17;
    L_B16: // isect_triangle_mid3
        fresh = false;
        if constexpr(kProf) count_block(ctx, 16, 7u);
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r42, R.r45, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r43, R.r46, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r44, R.r47, bitcast<float>(R.r14))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r58)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r58)) > static_cast<float>((0x0.0p+0f))));
        goto L_B17;
    L_B17: // isect_triangle_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 17, 7u);
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r58)) < static_cast<float>(R.r36))));
        R.r36 = static_cast<float>(((R.r54) ? (bitcast<float>(R.r58)) : (R.r36)));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r38) + static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r37 = static_cast<unsigned int>(((R.r54) ? (R.r10) : (R.r37)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r38) == static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r38 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r38) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        if(R.r14) goto L_B18; else goto L_B13;
    L_B18: // traverse_sphere
        fresh = false;
        if constexpr(kProf) count_block(ctx, 18, 25u);
        R.r33 = static_cast<float>((0x1.99999a0000000p-4f));
        R.r34 = static_cast<float>((-0x1.6666660000000p-1f));
        R.r35 = static_cast<float>((0x1.3333340000000p-2f));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r33)));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r34)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r35)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.3333340000000p-2f)) * static_cast<float>((0x1.3333340000000p-2f)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r42, R.r42, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r43, R.r43, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r44, R.r44, bitcast<float>(R.r10))));
        R.r41 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) - static_cast<float>(bitcast<float>(R.r14))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r43) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r44) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r40 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r40 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r42, bitcast<float>(R.r40))));
        R.r40 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r43, bitcast<float>(R.r40))));
        R.r40 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r32, R.r44, bitcast<float>(R.r40))));
        R.r39 = static_cast<float>((0x0.0p+0f));
        R.r39 = static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), R.r39));
        R.r39 = static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), R.r39));
        R.r39 = static_cast<float>(op_fma(R.r32, R.r32, R.r39));
        R.r38 = static_cast<unsigned int>(((unsigned int)0x8ull));
        goto L_B19;
    L_B19: // traverse_solve_quadratic
        if(budget == 0u) return 19;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 19, 3u);
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(R.r39))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r54)) > static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r54) goto L_B22; else goto L_B20;
    L_B20: // sq_head1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 20, 3u);
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r40)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r54)) > static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r54) goto L_B21; else goto L_B26;
    L_B21: // sq_head2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 21, 3u);
        R.r58 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(-static_cast<float>(R.r41))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r58)) / static_cast<float>(bitcast<float>(R.r40)))));
        goto L_B26;
    L_B22: // sq_mid1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 22, 5u);
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r41) * static_cast<float>(R.r39))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>((0x1.0000000000000p+2f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r40), bitcast<float>(R.r40), (-(bitcast<float>(R.r14))))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r54) goto L_B23; else goto L_B26;
    L_B23: // sq_mid2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 23, 11u);
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r58 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r40)) < static_cast<float>((0x0.0p+0f))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r40)) - static_cast<float>(bitcast<float>(R.r54)))));
        R.r40 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r40)) + static_cast<float>(bitcast<float>(R.r54)))));
        R.r40 = bitcast<unsigned int>(static_cast<float>(((R.r58) ? (bitcast<float>(R.r10)) : (bitcast<float>(R.r40)))));
        R.r40 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r40)) * static_cast<float>((-0x1.0000000000000p-1f)))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r40)) / static_cast<float>(R.r39))));
        R.r41 = static_cast<float>(static_cast<float>(static_cast<float>(R.r41) / static_cast<float>(bitcast<float>(R.r40))));
        R.r40 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r58)) < static_cast<float>((0x0.0p+0f))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(((R.r40) ? (R.r41) : (bitcast<float>(R.r58)))));
        if(R.r40) goto L_B25; else goto L_B24;
    L_B24: // sq_mid
        fresh = false;
        if constexpr(kProf) count_block(ctx, 24, 4u);
        R.r40 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r41) < static_cast<float>((0x0.0p+0f))));
        R.r54 = bitcast<unsigned int>(static_cast<float>(op_min<float>(static_cast<float>(bitcast<float>(R.r58)), static_cast<float>(R.r41))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(((R.r40) ? (bitcast<float>(R.r58)) : (bitcast<float>(R.r54)))));
        goto L_B25;
    L_B25: // sq_tail
        fresh = false;
        if constexpr(kProf) count_block(ctx, 25, 3u);
        R.r54 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r58)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r54)) >= static_cast<float>((0x0.0p+0f))));
        goto L_B26;
    L_B26: // sq_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 26, 2u);
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r38) == static_cast<unsigned int>(((unsigned int)0x8ull))));
        if(R.r14) goto L_B27; else goto L_B29;
    L_B27: // traverse_sphere_fin
        fresh = false;
        if constexpr(kProf) count_block(ctx, 27, 4u);
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r58)) < static_cast<float>(R.r36))));
        R.r36 = static_cast<float>(((R.r54) ? (bitcast<float>(R.r58)) : (R.r36)));
        R.r37 = static_cast<unsigned int>(((R.r54) ? (R.r38) : (R.r37)));
        goto L_B28;
    L_B28: // traverse_cylinder
        fresh = false;
        if constexpr(kProf) count_block(ctx, 28, 13u);
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>((-0x1.0000000000000p+0f))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>((-0x1.3333340000000p-2f))));
        R.r39 = static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(R.r32)));
        R.r39 = static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), R.r39));
        R.r40 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(R.r32))));
        R.r40 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r33, bitcast<float>(R.r6), bitcast<float>(R.r40))));
        R.r40 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r40)) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r41 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p-2f)) * static_cast<float>((0x1.0000000000000p-2f))));
        R.r41 = static_cast<float>(op_fma(R.r35, R.r35, (-(R.r41))));
        R.r41 = static_cast<float>(op_fma(R.r33, R.r33, R.r41));
        R.r38 = static_cast<unsigned int>(((unsigned int)0x9ull));
        goto L_B19;
    L_B29: // traverse_cylinder_fin
        fresh = false;
        if constexpr(kProf) count_block(ctx, 29, 15u);
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r58), R.r34)));
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x0.0p+0f)))));
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) <= static_cast<float>((0x1.4ccccc0000000p-1f)))));
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r58)) < static_cast<float>(R.r36))));
        R.r36 = static_cast<float>(((R.r54) ? (bitcast<float>(R.r58)) : (R.r36)));
        R.r37 = static_cast<unsigned int>(((R.r54) ? (R.r38) : (R.r37)));
        R.r38 = static_cast<unsigned int>(((unsigned int)0xaull));
        R.r33 = static_cast<float>((0x1.0000000000000p-1f));
        R.r34 = static_cast<float>((-0x1.6666660000000p-2f));
        R.r35 = static_cast<float>((-0x1.3333340000000p-2f));
        R.r39 = static_cast<float>((0x0.0p+0f));
        R.r40 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p+0f)));
        R.r41 = static_cast<float>((0x0.0p+0f));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p-2f)));
        goto L_B30;
    L_B30: // traverse_disk
        if(budget == 0u) return 30;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 30, 14u);
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) - static_cast<float>(R.r22)));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r34) - static_cast<float>(R.r23)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) - static_cast<float>(R.r24)));
        R.r58 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r42, R.r39, bitcast<float>(R.r58))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r43, bitcast<float>(R.r40), bitcast<float>(R.r58))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r44, R.r41, bitcast<float>(R.r58))));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r39, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r40), bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r32, R.r41, bitcast<float>(R.r10))));
        R.r58 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r58)) / static_cast<float>(bitcast<float>(R.r10)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r58)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r54) goto L_B31; else goto L_B32;
    L_B31: // isect_disk_rest
        fresh = false;
        if constexpr(kProf) count_block(ctx, 31, 16u);
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r58))));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r58))));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(bitcast<float>(R.r58))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) + static_cast<float>(R.r22)));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r43) + static_cast<float>(R.r23)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r44) + static_cast<float>(R.r24)));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r33)));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r43) - static_cast<float>(R.r34)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r44) - static_cast<float>(R.r35)));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r42, R.r42, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r43, R.r43, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r44, R.r44, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r10)))));
        R.r54 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r10)) < static_cast<float>(bitcast<float>(R.r14))));
        goto L_B32;
    L_B32: // isect_disk_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 32, 13u);
        R.r54 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r58)) < static_cast<float>(R.r36))));
        R.r36 = static_cast<float>(((R.r54) ? (bitcast<float>(R.r58)) : (R.r36)));
        R.r37 = static_cast<unsigned int>(((R.r54) ? (R.r38) : (R.r37)));
        R.r10 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r38) == static_cast<unsigned int>(((unsigned int)0xbull))));
        R.r38 = static_cast<unsigned int>(((unsigned int)0xbull));
        R.r33 = static_cast<float>((0x0.0p+0f));
        R.r34 = static_cast<float>((0x1.fff2e40000000p-1f));
        R.r35 = static_cast<float>((0x0.0p+0f));
        R.r39 = static_cast<float>((0x0.0p+0f));
        R.r40 = bitcast<unsigned int>(static_cast<float>((-0x1.0000000000000p+0f)));
        R.r41 = static_cast<float>((0x0.0p+0f));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x1.6666660000000p-2f)));
        if(R.r10) goto L_B33; else goto L_B30;
    L_B33: // traverse_room_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 33, 2u);
        R.r5 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r5) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        goto L_B34;
    L_B34: // radiance
        fresh = false;
        if constexpr(kProf) count_block(ctx, 34, 10u);
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0xbull))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(((R.r14) ? ((0x1.4000000000000p+2f)) : ((0x1.0000000000000p+0f)))));
        R.r11 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0xcull))));
        R.r11 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r11) || static_cast<unsigned int>(static_cast<unsigned int>(R.r31) >= static_cast<unsigned int>(((unsigned int)0x2ull)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(((R.r11) ? ((0x0.0p+0f)) : (bitcast<float>(R.r10)))));
        R.r25 = static_cast<float>(static_cast<float>(static_cast<float>(R.r25) * static_cast<float>(bitcast<float>(R.r10))));
        R.r26 = static_cast<float>(static_cast<float>(static_cast<float>(R.r26) * static_cast<float>(bitcast<float>(R.r10))));
        R.r27 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(bitcast<float>(R.r10))));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r14) || static_cast<unsigned int>(R.r11)));
        if(R.r14) goto L_B42; else goto L_B35;
    L_B35: // set_materials
        if(stop_heavy && !fresh) return 35;
    L_B35_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 35, 31u);
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r36)));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r36)));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(R.r36)));
        R.r22 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) + static_cast<float>(R.r33)));
        R.r23 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) + static_cast<float>(R.r34)));
        R.r24 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) + static_cast<float>(R.r35)));
        R.r14 = static_cast<unsigned int>(op_min<unsigned int>(static_cast<unsigned int>(R.r37), static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r28 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.0000000000000p+0f) : ((R.r14) == 1 ? (0x1.0000000000000p+0f) : ((R.r14) == 2 ? (0x1.99999a0000000p-3f) : ((R.r14) == 3 ? (0x1.0000000000000p+0f) : ((R.r14) == 4 ? (0x1.0000000000000p+0f) : (0x0.0p+0f))))))));
        R.r29 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.0000000000000p+0f) : ((R.r14) == 1 ? (0x1.99999a0000000p-2f) : ((R.r14) == 2 ? (0x1.0000000000000p+0f) : ((R.r14) == 3 ? (0x1.0000000000000p+0f) : ((R.r14) == 4 ? (0x1.0000000000000p+0f) : (0x1.b22d100000000p-3f))))))));
        R.r30 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.0000000000000p+0f) : ((R.r14) == 1 ? (0x1.99999a0000000p-3f) : ((R.r14) == 2 ? (0x1.99999a0000000p-2f) : ((R.r14) == 3 ? (0x1.0000000000000p+0f) : ((R.r14) == 4 ? (0x1.0000000000000p+0f) : (0x1.1b22d20000000p-1f))))))));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r28 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : (R.r28)));
        R.r29 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : (R.r29)));
        R.r30 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : (R.r30)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) || static_cast<unsigned int>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0xaull)))));
        R.r28 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : (R.r28)));
        R.r29 = static_cast<float>(((R.r14) ? ((0x1.a76c8c0000000p-1f)) : (R.r29)));
        R.r30 = static_cast<float>(((R.r14) ? ((0x1.12f1aa0000000p-1f)) : (R.r30)));
        R.r59 = static_cast<float>((0x0.0p+0f));
        R.r60 = static_cast<float>((0x1.0000000000000p+0f));
        R.r61 = static_cast<float>((0x0.0p+0f));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0xaull))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) || static_cast<unsigned int>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0xbull)))));
        R.r10 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) || static_cast<unsigned int>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0x9ull)))));
        R.r38 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r38 = static_cast<unsigned int>(((R.r14) ? (((unsigned int)0x1ull)) : (R.r38)));
        R.r11 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r37) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r38 = static_cast<unsigned int>(((R.r10) ? (R.r11) : (R.r38)));
        switch(R.r38) {
        case 0: goto L_B36;
        case 1: goto L_B37;
        case 2: goto L_B38;
        case 3: goto L_B39;
        default: goto L_HALT;
        }
    L_B36: // set_polygon_normal
        fresh = false;
        if constexpr(kProf) count_block(ctx, 36, 4u);
        R.r62 = static_cast<float>(static_cast<float>(((R.r37) == 0 ? (0x0.0p+0f) : ((R.r37) == 1 ? (0x1.0000000000000p+0f) : ((R.r37) == 2 ? (-0x1.0000000000000p+0f) : ((R.r37) == 3 ? (0x0.0p+0f) : ((R.r37) == 4 ? (0x0.0p+0f) : ((R.r37) == 5 ? (-0x1.d52cd80000000p-1f) : ((R.r37) == 6 ? (0x1.5775c60000000p-1f) : (0x1.f6dc440000000p-3f))))))))));
        R.r63 = static_cast<float>(static_cast<float>(((R.r37) == 0 ? (0x1.0000000000000p+0f) : ((R.r37) == 1 ? (0x0.0p+0f) : ((R.r37) == 2 ? (0x0.0p+0f) : ((R.r37) == 3 ? (-0x1.0000000000000p+0f) : ((R.r37) == 4 ? (0x0.0p+0f) : ((R.r37) == 5 ? (0x1.43d1320000000p-2f) : ((R.r37) == 6 ? (0x1.43d1360000000p-2f) : (0x1.43d1360000000p-2f))))))))));
        R.r64 = static_cast<float>(static_cast<float>(((R.r37) == 0 ? (0x0.0p+0f) : ((R.r37) == 1 ? (0x0.0p+0f) : ((R.r37) == 2 ? (0x0.0p+0f) : ((R.r37) == 3 ? (0x0.0p+0f) : ((R.r37) == 4 ? (0x1.0000000000000p+0f) : ((R.r37) == 5 ? (0x1.f6dc380000000p-3f) : ((R.r37) == 6 ? (0x1.5775c60000000p-1f) : (-0x1.d52cd40000000p-1f))))))))));
        goto L_B40;
    L_B37: // set_disk_normal
        fresh = false;
        if constexpr(kProf) count_block(ctx, 37, 19u);
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r37) == static_cast<unsigned int>(((unsigned int)0xaull))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>((-0x1.6666660000000p-2f))));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>((-0x1.3333340000000p-2f))));
        R.r10 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r42, R.r42, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r43, R.r43, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r44, R.r44, bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r10)))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) * static_cast<float>(bitcast<float>(R.r10))));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r43) * static_cast<float>(bitcast<float>(R.r10))));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r44) * static_cast<float>(bitcast<float>(R.r10))));
        R.r62 = static_cast<float>((0x0.0p+0f));
        R.r63 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : ((-0x1.0000000000000p+0f))));
        R.r64 = static_cast<float>((0x0.0p+0f));
        R.r59 = static_cast<float>(((R.r14) ? (R.r42) : (R.r59)));
        R.r60 = static_cast<float>(((R.r14) ? (R.r43) : (R.r60)));
        R.r61 = static_cast<float>(((R.r14) ? (R.r44) : (R.r61)));
        goto L_B40;
    L_B38: // compute_sphere_normal
        fresh = false;
        if constexpr(kProf) count_block(ctx, 38, 12u);
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>((0x1.99999a0000000p-4f))));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>((-0x1.6666660000000p-1f))));
        R.r64 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>((0x1.3333340000000p-2f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r62, R.r62, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r63, R.r63, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r64, R.r64, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r62) * static_cast<float>(bitcast<float>(R.r14))));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r63) * static_cast<float>(bitcast<float>(R.r14))));
        R.r64 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) * static_cast<float>(bitcast<float>(R.r14))));
        goto L_B40;
    L_B39: // compute_cylinder_normal
        fresh = false;
        if constexpr(kProf) count_block(ctx, 39, 12u);
        R.r63 = static_cast<float>((0x0.0p+0f));
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r64 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>((-0x1.3333340000000p-2f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r62, R.r62, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r63, R.r63, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r64, R.r64, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r62) * static_cast<float>(bitcast<float>(R.r14))));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r63) * static_cast<float>(bitcast<float>(R.r14))));
        R.r64 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) * static_cast<float>(bitcast<float>(R.r14))));
        goto L_B40;
    L_B40: // set_materials_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 40, 2u);
        R.r18 = static_cast<unsigned int>(((unsigned int)0x2ull));
        goto L_B1;
    L_B41: // lambert_indirect
        if(stop_heavy && !fresh) return 41;
    L_B41_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 41, 70u);
        R.r61 = static_cast<float>(op_copysign(static_cast<float>((0x1.0000000000000p+0f)), static_cast<float>(R.r64)));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r61) + static_cast<float>(R.r64)));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>((-0x1.0000000000000p+0f)) / static_cast<float>(R.r33)));
        R.r59 = static_cast<float>(static_cast<float>(static_cast<float>(R.r62) * static_cast<float>(R.r63)));
        R.r59 = static_cast<float>(static_cast<float>(static_cast<float>(R.r59) * static_cast<float>(R.r33)));
        R.r60 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) * static_cast<float>(R.r63)));
        R.r60 = static_cast<float>(static_cast<float>(static_cast<float>(R.r60) * static_cast<float>(R.r63)));
        R.r60 = static_cast<float>(static_cast<float>(static_cast<float>(R.r60) + static_cast<float>(R.r61)));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) * static_cast<float>(R.r62)));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) * static_cast<float>(R.r62)));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) * static_cast<float>(R.r61)));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) + static_cast<float>((0x1.0000000000000p+0f))));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(R.r61) * static_cast<float>(R.r59)));
        R.r35 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r61)));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(R.r62)));
        R.r61 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r63)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r33, R.r33, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r34, R.r34, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r35, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) * static_cast<float>(bitcast<float>(R.r14))));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(R.r34) * static_cast<float>(bitcast<float>(R.r14))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r59, R.r59, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r60, R.r60, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r61, R.r61, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r59 = static_cast<float>(static_cast<float>(static_cast<float>(R.r59) * static_cast<float>(bitcast<float>(R.r14))));
        R.r60 = static_cast<float>(static_cast<float>(static_cast<float>(R.r60) * static_cast<float>(bitcast<float>(R.r14))));
        R.r61 = static_cast<float>(static_cast<float>(static_cast<float>(R.r61) * static_cast<float>(bitcast<float>(R.r14))));
        R.r20 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) - static_cast<float>((0x1.0000000000000p-1f)))));
        R.r20 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) * static_cast<float>((0x1.921fb60000000p+2f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r21)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_cos(static_cast<float>(bitcast<float>(R.r20)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) * static_cast<float>(bitcast<float>(R.r10))));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(R.r34) * static_cast<float>(bitcast<float>(R.r10))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r10))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_sin(static_cast<float>(bitcast<float>(R.r20)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r59 = static_cast<float>(static_cast<float>(static_cast<float>(R.r59) * static_cast<float>(bitcast<float>(R.r10))));
        R.r60 = static_cast<float>(static_cast<float>(static_cast<float>(R.r60) * static_cast<float>(bitcast<float>(R.r10))));
        R.r61 = static_cast<float>(static_cast<float>(static_cast<float>(R.r61) * static_cast<float>(bitcast<float>(R.r10))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r21)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r62) * static_cast<float>(bitcast<float>(R.r14))));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r63) * static_cast<float>(bitcast<float>(R.r14))));
        R.r64 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) * static_cast<float>(bitcast<float>(R.r14))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r33) + static_cast<float>(R.r59))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r34) + static_cast<float>(R.r60))));
        R.r32 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) + static_cast<float>(R.r61)));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) + static_cast<float>(R.r62))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) + static_cast<float>(R.r63))));
        R.r32 = static_cast<float>(static_cast<float>(static_cast<float>(R.r32) + static_cast<float>(R.r64)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r32, R.r32, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r32 = static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(bitcast<float>(R.r14))));
        R.r25 = static_cast<float>(static_cast<float>(static_cast<float>(R.r25) * static_cast<float>(R.r28)));
        R.r26 = static_cast<float>(static_cast<float>(static_cast<float>(R.r26) * static_cast<float>(R.r29)));
        R.r27 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r30)));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r31 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r31) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        goto L_B3;
    L_B42: // fin_sample
        fresh = false;
        if constexpr(kProf) count_block(ctx, 42, 23u);
        R.r2 = static_cast<float>(static_cast<float>(static_cast<float>(R.r2) + static_cast<float>(R.r25)));
        R.r3 = static_cast<float>(static_cast<float>(static_cast<float>(R.r3) + static_cast<float>(R.r26)));
        R.r4 = static_cast<float>(static_cast<float>(static_cast<float>(R.r4) + static_cast<float>(R.r27)));
        R.r11 = bitcast<unsigned int>(static_cast<float>(R.r19));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r25, (0x1.b367a00000000p-3f), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r26, (0x1.6e2eb20000000p-1f), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r27, (0x1.27bb300000000p-4f), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_min<float>(static_cast<float>(bitcast<float>(R.r14)), static_cast<float>((0x1.0000000000000p+0f)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) - static_cast<float>(R.r16))));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) / static_cast<float>(bitcast<float>(R.r11))));
        R.r16 = static_cast<float>(static_cast<float>(static_cast<float>(R.r16) + static_cast<float>(R.r33)));
        R.r34 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) - static_cast<float>(R.r16)));
        R.r17 = static_cast<float>(op_fma(bitcast<float>(R.r10), R.r34, R.r17));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) - static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(R.r10));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r17) / static_cast<float>(bitcast<float>(R.r10)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r10)))));
        R.r10 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r10)) / static_cast<float>(bitcast<float>(R.r11)))));
        R.r10 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r10)) < static_cast<float>((0x1.a36e2e0000000p-14f))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) && static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >= static_cast<unsigned int>(((unsigned int)0x40ull)))));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x0ull));
        if(R.r14) goto L_B43; else goto L_B1;
    L_B43: // fin_pixel
        fresh = false;
        if constexpr(kProf) count_block(ctx, 43, 5u);
        R.r19 = bitcast<unsigned int>(static_cast<float>(R.r19));
        R.r2 = static_cast<float>(static_cast<float>(static_cast<float>(R.r2) / static_cast<float>(bitcast<float>(R.r19))));
        R.r3 = static_cast<float>(static_cast<float>(static_cast<float>(R.r3) / static_cast<float>(bitcast<float>(R.r19))));
        R.r4 = static_cast<float>(static_cast<float>(static_cast<float>(R.r4) / static_cast<float>(bitcast<float>(R.r19))));
        goto L_HALT;
    L_HALT:
        return kHalt;
    }

    static constexpr unsigned long long kRowBytes = 6328ull;
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
                v0.y = bitcast<unsigned>(R.r22);
                v0.z = bitcast<unsigned>(R.r23);
                v0.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 0ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r25);
                v1.y = bitcast<unsigned>(R.r26);
                v1.z = bitcast<unsigned>(R.r27);
                v1.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 16ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r29);
                v2.y = bitcast<unsigned>(R.r30);
                v2.z = bitcast<unsigned>(R.r31);
                v2.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 32ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r58);
                v3.y = bitcast<unsigned>(R.r62);
                v3.z = bitcast<unsigned>(R.r63);
                v3.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 48ull * cap)[idx] = v3;
            }
            {
                unsigned v4;
                v4 = tid;
                reinterpret_cast<unsigned*>(base + 64ull * cap)[idx] = v4;
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
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 120ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 136ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 152ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 168ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r62);
                v7.y = bitcast<unsigned>(R.r63);
                v7.z = bitcast<unsigned>(R.r64);
                v7.w = tid;
                reinterpret_cast<uint4*>(base + 184ull * cap)[idx] = v7;
            }
            return;
        }
        case 2: // sample_pixel
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 200ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r8);
                v1.z = bitcast<unsigned>(R.r9);
                v1.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 216ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r13);
                v2.y = bitcast<unsigned>(R.r15);
                v2.z = bitcast<unsigned>(R.r16);
                v2.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 232ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r19);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 248ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r62);
                v4.y = bitcast<unsigned>(R.r63);
                v4.z = bitcast<unsigned>(R.r64);
                v4.w = tid;
                reinterpret_cast<uint4*>(base + 264ull * cap)[idx] = v4;
            }
            return;
        }
        case 3: // traverse_scene
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 280ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 296ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 312ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 328ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 344ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 360ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r58);
                v6.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 376ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r63);
                v7.y = bitcast<unsigned>(R.r64);
                v7.z = tid;
                reinterpret_cast<uint4*>(base + 392ull * cap)[idx] = v7;
            }
            return;
        }
        case 4: // traverse_box
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 408ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 424ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 440ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 456ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 472ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 488ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 504ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r58);
                v7.z = bitcast<unsigned>(R.r62);
                v7.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 520ull * cap)[idx] = v7;
            }
            {
                uint2 v8;
                v8.x = bitcast<unsigned>(R.r64);
                v8.y = tid;
                reinterpret_cast<uint2*>(base + 536ull * cap)[idx] = v8;
            }
            return;
        }
        case 5: // isect_quad_l1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 544ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 560ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 576ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 592ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 608ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 624ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 640ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r36);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 656ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r38);
                v8.y = bitcast<unsigned>(R.r39);
                v8.z = bitcast<unsigned>(R.r40);
                v8.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 672ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r42);
                v9.y = bitcast<unsigned>(R.r43);
                v9.z = bitcast<unsigned>(R.r44);
                v9.w = bitcast<unsigned>(R.r45);
                reinterpret_cast<uint4*>(base + 688ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r46);
                v10.y = bitcast<unsigned>(R.r47);
                v10.z = bitcast<unsigned>(R.r55);
                v10.w = bitcast<unsigned>(R.r56);
                reinterpret_cast<uint4*>(base + 704ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r57);
                v11.y = bitcast<unsigned>(R.r58);
                v11.z = bitcast<unsigned>(R.r62);
                v11.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 720ull * cap)[idx] = v11;
            }
            {
                uint2 v12;
                v12.x = bitcast<unsigned>(R.r64);
                v12.y = tid;
                reinterpret_cast<uint2*>(base + 736ull * cap)[idx] = v12;
            }
            return;
        }
        case 6: // isect_quad_l2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 744ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 760ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r10);
                v2.z = bitcast<unsigned>(R.r12);
                v2.w = bitcast<unsigned>(R.r13);
                reinterpret_cast<uint4*>(base + 776ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r14);
                v3.y = bitcast<unsigned>(R.r15);
                v3.z = bitcast<unsigned>(R.r16);
                v3.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 792ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 808ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 824ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 840ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 856ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r39);
                v8.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 872ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r41);
                v9.y = bitcast<unsigned>(R.r42);
                v9.z = bitcast<unsigned>(R.r43);
                v9.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 888ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r45);
                v10.y = bitcast<unsigned>(R.r46);
                v10.z = bitcast<unsigned>(R.r47);
                v10.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 904ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r62);
                v11.y = bitcast<unsigned>(R.r63);
                v11.z = bitcast<unsigned>(R.r64);
                v11.w = tid;
                reinterpret_cast<uint4*>(base + 920ull * cap)[idx] = v11;
            }
            return;
        }
        case 7: // isect_quad_l3
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 936ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 952ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r10);
                v2.z = bitcast<unsigned>(R.r11);
                v2.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 968ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r13);
                v3.y = bitcast<unsigned>(R.r14);
                v3.z = bitcast<unsigned>(R.r15);
                v3.w = bitcast<unsigned>(R.r16);
                reinterpret_cast<uint4*>(base + 984ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r17);
                v4.y = bitcast<unsigned>(R.r19);
                v4.z = bitcast<unsigned>(R.r22);
                v4.w = bitcast<unsigned>(R.r23);
                reinterpret_cast<uint4*>(base + 1000ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r24);
                v5.y = bitcast<unsigned>(R.r25);
                v5.z = bitcast<unsigned>(R.r26);
                v5.w = bitcast<unsigned>(R.r27);
                reinterpret_cast<uint4*>(base + 1016ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r28);
                v6.y = bitcast<unsigned>(R.r29);
                v6.z = bitcast<unsigned>(R.r30);
                v6.w = bitcast<unsigned>(R.r31);
                reinterpret_cast<uint4*>(base + 1032ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r32);
                v7.y = bitcast<unsigned>(R.r33);
                v7.z = bitcast<unsigned>(R.r34);
                v7.w = bitcast<unsigned>(R.r35);
                reinterpret_cast<uint4*>(base + 1048ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r36);
                v8.y = bitcast<unsigned>(R.r37);
                v8.z = bitcast<unsigned>(R.r38);
                v8.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 1064ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r40);
                v9.y = bitcast<unsigned>(R.r41);
                v9.z = bitcast<unsigned>(R.r42);
                v9.w = bitcast<unsigned>(R.r43);
                reinterpret_cast<uint4*>(base + 1080ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r44);
                v10.y = bitcast<unsigned>(R.r45);
                v10.z = bitcast<unsigned>(R.r46);
                v10.w = bitcast<unsigned>(R.r47);
                reinterpret_cast<uint4*>(base + 1096ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r62);
                v11.y = bitcast<unsigned>(R.r63);
                v11.z = bitcast<unsigned>(R.r64);
                v11.w = tid;
                reinterpret_cast<uint4*>(base + 1112ull * cap)[idx] = v11;
            }
            return;
        }
        case 8: // isect_quad_l4
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1128ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1144ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 1160ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 1176ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 1192ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 1208ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1224ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r36);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 1240ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r38);
                v8.y = bitcast<unsigned>(R.r39);
                v8.z = bitcast<unsigned>(R.r40);
                v8.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 1256ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r42);
                v9.y = bitcast<unsigned>(R.r43);
                v9.z = bitcast<unsigned>(R.r44);
                v9.w = bitcast<unsigned>(R.r45);
                reinterpret_cast<uint4*>(base + 1272ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r46);
                v10.y = bitcast<unsigned>(R.r47);
                v10.z = bitcast<unsigned>(R.r62);
                v10.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 1288ull * cap)[idx] = v10;
            }
            {
                uint2 v11;
                v11.x = bitcast<unsigned>(R.r64);
                v11.y = tid;
                reinterpret_cast<uint2*>(base + 1304ull * cap)[idx] = v11;
            }
            return;
        }
        case 9: // isect_quad_l5
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1312ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1328ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 1344ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 1360ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 1376ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 1392ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1408ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r36);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 1424ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r38);
                v8.y = bitcast<unsigned>(R.r39);
                v8.z = bitcast<unsigned>(R.r40);
                v8.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 1440ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r42);
                v9.y = bitcast<unsigned>(R.r43);
                v9.z = bitcast<unsigned>(R.r44);
                v9.w = bitcast<unsigned>(R.r45);
                reinterpret_cast<uint4*>(base + 1456ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r46);
                v10.y = bitcast<unsigned>(R.r47);
                v10.z = bitcast<unsigned>(R.r48);
                v10.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 1472ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r50);
                v11.y = bitcast<unsigned>(R.r55);
                v11.z = bitcast<unsigned>(R.r56);
                v11.w = bitcast<unsigned>(R.r57);
                reinterpret_cast<uint4*>(base + 1488ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r58);
                v12.y = bitcast<unsigned>(R.r62);
                v12.z = bitcast<unsigned>(R.r63);
                v12.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 1504ull * cap)[idx] = v12;
            }
            {
                unsigned v13;
                v13 = tid;
                reinterpret_cast<unsigned*>(base + 1520ull * cap)[idx] = v13;
            }
            return;
        }
        case 10: // isect_quad_l6
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1528ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1544ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 1560ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 1576ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 1592ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 1608ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1624ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r36);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 1640ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r38);
                v8.y = bitcast<unsigned>(R.r39);
                v8.z = bitcast<unsigned>(R.r40);
                v8.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 1656ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r45);
                v9.y = bitcast<unsigned>(R.r46);
                v9.z = bitcast<unsigned>(R.r47);
                v9.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 1672ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r49);
                v10.y = bitcast<unsigned>(R.r50);
                v10.z = bitcast<unsigned>(R.r51);
                v10.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 1688ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r53);
                v11.y = bitcast<unsigned>(R.r58);
                v11.z = bitcast<unsigned>(R.r62);
                v11.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 1704ull * cap)[idx] = v11;
            }
            {
                uint2 v12;
                v12.x = bitcast<unsigned>(R.r64);
                v12.y = tid;
                reinterpret_cast<uint2*>(base + 1720ull * cap)[idx] = v12;
            }
            return;
        }
        case 11: // isect_quad_l7
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1728ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1744ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 1760ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 1776ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 1792ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 1808ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 1824ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r36);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 1840ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r38);
                v8.y = bitcast<unsigned>(R.r39);
                v8.z = bitcast<unsigned>(R.r40);
                v8.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 1856ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r45);
                v9.y = bitcast<unsigned>(R.r46);
                v9.z = bitcast<unsigned>(R.r47);
                v9.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 1872ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r63);
                v10.y = bitcast<unsigned>(R.r64);
                v10.z = tid;
                reinterpret_cast<uint4*>(base + 1888ull * cap)[idx] = v10;
            }
            return;
        }
        case 12: // isect_quad_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1904ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1920ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 1936ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 1952ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 1968ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 1984ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 2000ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r54);
                v7.z = bitcast<unsigned>(R.r58);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 2016ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = tid;
                reinterpret_cast<uint4*>(base + 2032ull * cap)[idx] = v8;
            }
            return;
        }
        case 13: // traverse_tetrahedron
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2048ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2064ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2080ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2096ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 2112ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 2128ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 2144ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r62);
                v7.z = bitcast<unsigned>(R.r63);
                v7.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 2160ull * cap)[idx] = v7;
            }
            {
                unsigned v8;
                v8 = tid;
                reinterpret_cast<unsigned*>(base + 2176ull * cap)[idx] = v8;
            }
            return;
        }
        case 14: // isect_triangle_mid1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2184ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2200ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2216ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2232ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 2248ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 2264ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 2280ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r35);
                v7.y = bitcast<unsigned>(R.r36);
                v7.z = bitcast<unsigned>(R.r37);
                v7.w = bitcast<unsigned>(R.r38);
                reinterpret_cast<uint4*>(base + 2296ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r39);
                v8.y = bitcast<unsigned>(R.r40);
                v8.z = bitcast<unsigned>(R.r41);
                v8.w = bitcast<unsigned>(R.r42);
                reinterpret_cast<uint4*>(base + 2312ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r43);
                v9.y = bitcast<unsigned>(R.r44);
                v9.z = bitcast<unsigned>(R.r45);
                v9.w = bitcast<unsigned>(R.r46);
                reinterpret_cast<uint4*>(base + 2328ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r47);
                v10.y = bitcast<unsigned>(R.r58);
                v10.z = bitcast<unsigned>(R.r62);
                v10.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 2344ull * cap)[idx] = v10;
            }
            {
                uint2 v11;
                v11.x = bitcast<unsigned>(R.r64);
                v11.y = tid;
                reinterpret_cast<uint2*>(base + 2360ull * cap)[idx] = v11;
            }
            return;
        }
        case 15: // isect_triangle_mid2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2368ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2384ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 2400ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 2416ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 2432ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 2448ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 2464ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r36);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 2480ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r38);
                v8.y = bitcast<unsigned>(R.r39);
                v8.z = bitcast<unsigned>(R.r40);
                v8.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 2496ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r42);
                v9.y = bitcast<unsigned>(R.r43);
                v9.z = bitcast<unsigned>(R.r44);
                v9.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 2512ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r62);
                v10.y = bitcast<unsigned>(R.r63);
                v10.z = bitcast<unsigned>(R.r64);
                v10.w = tid;
                reinterpret_cast<uint4*>(base + 2528ull * cap)[idx] = v10;
            }
            return;
        }
        case 16: // isect_triangle_mid3
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2544ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2560ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2576ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2592ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 2608ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 2624ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 2640ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r42);
                v7.z = bitcast<unsigned>(R.r43);
                v7.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 2656ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r45);
                v8.y = bitcast<unsigned>(R.r46);
                v8.z = bitcast<unsigned>(R.r47);
                v8.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 2672ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r62);
                v9.y = bitcast<unsigned>(R.r63);
                v9.z = bitcast<unsigned>(R.r64);
                v9.w = tid;
                reinterpret_cast<uint4*>(base + 2688ull * cap)[idx] = v9;
            }
            return;
        }
        case 17: // isect_triangle_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2704ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2720ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2736ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2752ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 2768ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 2784ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 2800ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r54);
                v7.z = bitcast<unsigned>(R.r58);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 2816ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = tid;
                reinterpret_cast<uint4*>(base + 2832ull * cap)[idx] = v8;
            }
            return;
        }
        case 18: // traverse_sphere
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2848ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 2864ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2880ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2896ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 2912ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 2928ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 2944ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r58);
                v7.y = bitcast<unsigned>(R.r62);
                v7.z = bitcast<unsigned>(R.r63);
                v7.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 2960ull * cap)[idx] = v7;
            }
            {
                unsigned v8;
                v8 = tid;
                reinterpret_cast<unsigned*>(base + 2976ull * cap)[idx] = v8;
            }
            return;
        }
        case 19: // traverse_solve_quadratic
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2984ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 3000ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 3016ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 3032ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 3048ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 3064ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r34);
                v6.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 3080ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r37);
                v7.y = bitcast<unsigned>(R.r38);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 3096ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r58);
                v8.z = bitcast<unsigned>(R.r62);
                v8.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 3112ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r64);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 3128ull * cap)[idx] = v9;
            }
            return;
        }
        case 20: // sq_head1
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
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 3168ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 3184ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 3200ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 3216ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r34);
                v6.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 3232ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r37);
                v7.y = bitcast<unsigned>(R.r38);
                v7.z = bitcast<unsigned>(R.r40);
                v7.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 3248ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r58);
                v8.y = bitcast<unsigned>(R.r62);
                v8.z = bitcast<unsigned>(R.r63);
                v8.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 3264ull * cap)[idx] = v8;
            }
            {
                unsigned v9;
                v9 = tid;
                reinterpret_cast<unsigned*>(base + 3280ull * cap)[idx] = v9;
            }
            return;
        }
        case 21: // sq_head2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3288ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 3304ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 3320ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 3336ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 3352ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 3368ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r34);
                v6.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 3384ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r37);
                v7.y = bitcast<unsigned>(R.r38);
                v7.z = bitcast<unsigned>(R.r40);
                v7.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 3400ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r54);
                v8.y = bitcast<unsigned>(R.r62);
                v8.z = bitcast<unsigned>(R.r63);
                v8.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 3416ull * cap)[idx] = v8;
            }
            {
                unsigned v9;
                v9 = tid;
                reinterpret_cast<unsigned*>(base + 3432ull * cap)[idx] = v9;
            }
            return;
        }
        case 22: // sq_mid1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3440ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 3456ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 3472ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 3488ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 3504ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 3520ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r34);
                v6.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 3536ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r37);
                v7.y = bitcast<unsigned>(R.r38);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 3552ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r58);
                v8.z = bitcast<unsigned>(R.r62);
                v8.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 3568ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r64);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 3584ull * cap)[idx] = v9;
            }
            return;
        }
        case 23: // sq_mid2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3592ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 3608ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 3624ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 3640ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 3656ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 3672ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 3688ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r36);
                v7.y = bitcast<unsigned>(R.r37);
                v7.z = bitcast<unsigned>(R.r38);
                v7.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 3704ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r40);
                v8.y = bitcast<unsigned>(R.r41);
                v8.z = bitcast<unsigned>(R.r62);
                v8.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 3720ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r64);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 3736ull * cap)[idx] = v9;
            }
            return;
        }
        case 24: // sq_mid
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3744ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 3760ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 3776ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 3792ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 3808ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 3824ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 3840ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r36);
                v7.y = bitcast<unsigned>(R.r37);
                v7.z = bitcast<unsigned>(R.r38);
                v7.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 3856ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r58);
                v8.y = bitcast<unsigned>(R.r62);
                v8.z = bitcast<unsigned>(R.r63);
                v8.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 3872ull * cap)[idx] = v8;
            }
            {
                unsigned v9;
                v9 = tid;
                reinterpret_cast<unsigned*>(base + 3888ull * cap)[idx] = v9;
            }
            return;
        }
        case 25: // sq_tail
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3896ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 3912ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 3928ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 3944ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 3960ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 3976ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 3992ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r36);
                v7.y = bitcast<unsigned>(R.r37);
                v7.z = bitcast<unsigned>(R.r38);
                v7.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 4008ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r62);
                v8.y = bitcast<unsigned>(R.r63);
                v8.z = bitcast<unsigned>(R.r64);
                v8.w = tid;
                reinterpret_cast<uint4*>(base + 4024ull * cap)[idx] = v8;
            }
            return;
        }
        case 26: // sq_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4040ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 4056ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 4072ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 4088ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 4104ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 4120ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r34);
                v6.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 4136ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r37);
                v7.y = bitcast<unsigned>(R.r38);
                v7.z = bitcast<unsigned>(R.r54);
                v7.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 4152ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r62);
                v8.y = bitcast<unsigned>(R.r63);
                v8.z = bitcast<unsigned>(R.r64);
                v8.w = tid;
                reinterpret_cast<uint4*>(base + 4168ull * cap)[idx] = v8;
            }
            return;
        }
        case 27: // traverse_sphere_fin
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4184ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 4200ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 4216ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 4232ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 4248ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 4264ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 4280ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r54);
                v7.z = bitcast<unsigned>(R.r58);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 4296ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = tid;
                reinterpret_cast<uint4*>(base + 4312ull * cap)[idx] = v8;
            }
            return;
        }
        case 28: // traverse_cylinder
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4328ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 4344ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 4360ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 4376ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 4392ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 4408ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 4424ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r58);
                v7.y = bitcast<unsigned>(R.r62);
                v7.z = bitcast<unsigned>(R.r63);
                v7.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 4440ull * cap)[idx] = v7;
            }
            {
                unsigned v8;
                v8 = tid;
                reinterpret_cast<unsigned*>(base + 4456ull * cap)[idx] = v8;
            }
            return;
        }
        case 29: // traverse_cylinder_fin
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4464ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 4480ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 4496ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 4512ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 4528ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 4544ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r34);
                v6.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 4560ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r37);
                v7.y = bitcast<unsigned>(R.r38);
                v7.z = bitcast<unsigned>(R.r54);
                v7.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 4576ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r62);
                v8.y = bitcast<unsigned>(R.r63);
                v8.z = bitcast<unsigned>(R.r64);
                v8.w = tid;
                reinterpret_cast<uint4*>(base + 4592ull * cap)[idx] = v8;
            }
            return;
        }
        case 30: // traverse_disk
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4608ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 4624ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 4640ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 4656ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 4672ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 4688ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 4704ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r36);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 4720ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r38);
                v8.y = bitcast<unsigned>(R.r39);
                v8.z = bitcast<unsigned>(R.r40);
                v8.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 4736ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r62);
                v9.y = bitcast<unsigned>(R.r63);
                v9.z = bitcast<unsigned>(R.r64);
                v9.w = tid;
                reinterpret_cast<uint4*>(base + 4752ull * cap)[idx] = v9;
            }
            return;
        }
        case 31: // isect_disk_rest
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4768ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 4784ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 4800ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 4816ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 4832ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 4848ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 4864ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r36);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 4880ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r38);
                v8.y = bitcast<unsigned>(R.r58);
                v8.z = bitcast<unsigned>(R.r62);
                v8.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 4896ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r64);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 4912ull * cap)[idx] = v9;
            }
            return;
        }
        case 32: // isect_disk_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4920ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 4936ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 4952ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 4968ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 4984ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 5000ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 5016ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r38);
                v7.y = bitcast<unsigned>(R.r54);
                v7.z = bitcast<unsigned>(R.r58);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 5032ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = tid;
                reinterpret_cast<uint4*>(base + 5048ull * cap)[idx] = v8;
            }
            return;
        }
        case 33: // traverse_room_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5064ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 5080ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5096ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 5112ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 5128ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 5144ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 5160ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r58);
                v7.y = bitcast<unsigned>(R.r62);
                v7.z = bitcast<unsigned>(R.r63);
                v7.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 5176ull * cap)[idx] = v7;
            }
            {
                unsigned v8;
                v8 = tid;
                reinterpret_cast<unsigned*>(base + 5192ull * cap)[idx] = v8;
            }
            return;
        }
        case 34: // radiance
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5200ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 5216ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5232ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 5248ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 5264ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 5280ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r36);
                v6.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 5296ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r58);
                v7.y = bitcast<unsigned>(R.r62);
                v7.z = bitcast<unsigned>(R.r63);
                v7.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 5312ull * cap)[idx] = v7;
            }
            {
                unsigned v8;
                v8 = tid;
                reinterpret_cast<unsigned*>(base + 5328ull * cap)[idx] = v8;
            }
            return;
        }
        case 35: // set_materials
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5336ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 5352ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5368ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 5384ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 5400ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r31);
                v5.z = bitcast<unsigned>(R.r32);
                v5.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 5416ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r37);
                v6.y = bitcast<unsigned>(R.r58);
                v6.z = tid;
                reinterpret_cast<uint4*>(base + 5432ull * cap)[idx] = v6;
            }
            return;
        }
        case 36: // set_polygon_normal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5448ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 5464ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5480ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 5496ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 5512ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 5528ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r37);
                v6.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 5544ull * cap)[idx] = v6;
            }
            {
                unsigned v7;
                v7 = tid;
                reinterpret_cast<unsigned*>(base + 5560ull * cap)[idx] = v7;
            }
            return;
        }
        case 37: // set_disk_normal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5568ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 5584ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5600ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 5616ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 5632ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 5648ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r37);
                v6.w = bitcast<unsigned>(R.r58);
                reinterpret_cast<uint4*>(base + 5664ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r59);
                v7.y = bitcast<unsigned>(R.r60);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = tid;
                reinterpret_cast<uint4*>(base + 5680ull * cap)[idx] = v7;
            }
            return;
        }
        case 38: // compute_sphere_normal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5696ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 5712ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5728ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 5744ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 5760ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 5776ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r58);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 5792ull * cap)[idx] = v6;
            }
            return;
        }
        case 39: // compute_cylinder_normal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5808ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 5824ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5840ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 5856ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 5872ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 5888ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r58);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 5904ull * cap)[idx] = v6;
            }
            return;
        }
        case 40: // set_materials_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5920ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 5936ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5952ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 5968ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 5984ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 6000ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r58);
                v6.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 6016ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r63);
                v7.y = bitcast<unsigned>(R.r64);
                v7.z = tid;
                reinterpret_cast<uint4*>(base + 6032ull * cap)[idx] = v7;
            }
            return;
        }
        case 41: // lambert_indirect
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 6048ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r8);
                v1.z = bitcast<unsigned>(R.r9);
                v1.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 6064ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r13);
                v2.y = bitcast<unsigned>(R.r15);
                v2.z = bitcast<unsigned>(R.r16);
                v2.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 6080ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r19);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 6096ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 6112ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 6128ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r58);
                v6.z = bitcast<unsigned>(R.r62);
                v6.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 6144ull * cap)[idx] = v6;
            }
            {
                uint2 v7;
                v7.x = bitcast<unsigned>(R.r64);
                v7.y = tid;
                reinterpret_cast<uint2*>(base + 6160ull * cap)[idx] = v7;
            }
            return;
        }
        case 42: // fin_sample
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 6168ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 6184ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 6200ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 6216ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 6232ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 6248ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r58);
                v6.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 6264ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r63);
                v7.y = bitcast<unsigned>(R.r64);
                v7.z = tid;
                reinterpret_cast<uint4*>(base + 6280ull * cap)[idx] = v7;
            }
            return;
        }
        case 43: // fin_pixel
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 6296ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r19);
                v1.z = tid;
                reinterpret_cast<uint4*>(base + 6312ull * cap)[idx] = v1;
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
            R.r22 = bitcast<float>(v0.y);
            R.r23 = bitcast<float>(v0.z);
            R.r24 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 16ull * cap)[idx];
            R.r25 = bitcast<float>(v1.x);
            R.r26 = bitcast<float>(v1.y);
            R.r27 = bitcast<float>(v1.z);
            R.r28 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 32ull * cap)[idx];
            R.r29 = bitcast<float>(v2.x);
            R.r30 = bitcast<float>(v2.y);
            R.r31 = bitcast<unsigned int>(v2.z);
            R.r32 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 48ull * cap)[idx];
            R.r58 = bitcast<unsigned int>(v3.x);
            R.r62 = bitcast<float>(v3.y);
            R.r63 = bitcast<float>(v3.z);
            R.r64 = bitcast<float>(v3.w);
            const unsigned v4 = reinterpret_cast<const unsigned*>(base + 64ull * cap)[idx];
            return v4;
        }
        case 1: // roll
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 136ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 152ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 168ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r58 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 184ull * cap)[idx];
            R.r62 = bitcast<float>(v7.x);
            R.r63 = bitcast<float>(v7.y);
            R.r64 = bitcast<float>(v7.z);
            return v7.w;
        }
        case 2: // sample_pixel
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 200ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 216ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r8 = bitcast<unsigned int>(v1.y);
            R.r9 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 232ull * cap)[idx];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r16 = bitcast<float>(v2.z);
            R.r17 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 248ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<unsigned int>(v3.y);
            R.r21 = bitcast<unsigned int>(v3.z);
            R.r58 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 264ull * cap)[idx];
            R.r62 = bitcast<float>(v4.x);
            R.r63 = bitcast<float>(v4.y);
            R.r64 = bitcast<float>(v4.z);
            return v4.w;
        }
        case 3: // traverse_scene
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 280ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 296ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 312ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 328ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 344ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 360ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 376ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            R.r62 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 392ull * cap)[idx];
            R.r63 = bitcast<float>(v7.x);
            R.r64 = bitcast<float>(v7.y);
            return v7.z;
        }
        case 4: // traverse_box
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 408ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 424ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 440ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 456ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 472ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 488ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 504ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 520ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r58 = bitcast<unsigned int>(v7.y);
            R.r62 = bitcast<float>(v7.z);
            R.r63 = bitcast<float>(v7.w);
            const uint2 v8 = reinterpret_cast<const uint2*>(base + 536ull * cap)[idx];
            R.r64 = bitcast<float>(v8.x);
            return v8.y;
        }
        case 5: // isect_quad_l1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 544ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 560ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 576ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 592ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 608ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 624ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 640ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 656ull * cap)[idx];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 672ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 688ull * cap)[idx];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<float>(v9.y);
            R.r44 = bitcast<float>(v9.z);
            R.r45 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 704ull * cap)[idx];
            R.r46 = bitcast<float>(v10.x);
            R.r47 = bitcast<float>(v10.y);
            R.r55 = bitcast<float>(v10.z);
            R.r56 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 720ull * cap)[idx];
            R.r57 = bitcast<float>(v11.x);
            R.r58 = bitcast<unsigned int>(v11.y);
            R.r62 = bitcast<float>(v11.z);
            R.r63 = bitcast<float>(v11.w);
            const uint2 v12 = reinterpret_cast<const uint2*>(base + 736ull * cap)[idx];
            R.r64 = bitcast<float>(v12.x);
            return v12.y;
        }
        case 6: // isect_quad_l2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 744ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 760ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 776ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r12 = bitcast<float>(v2.z);
            R.r13 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 792ull * cap)[idx];
            R.r14 = bitcast<unsigned int>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r16 = bitcast<float>(v3.z);
            R.r17 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 808ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 824ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 840ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<unsigned int>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 856ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<float>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 872ull * cap)[idx];
            R.r37 = bitcast<unsigned int>(v8.x);
            R.r38 = bitcast<unsigned int>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 888ull * cap)[idx];
            R.r41 = bitcast<float>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<float>(v9.z);
            R.r44 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 904ull * cap)[idx];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r58 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 920ull * cap)[idx];
            R.r62 = bitcast<float>(v11.x);
            R.r63 = bitcast<float>(v11.y);
            R.r64 = bitcast<float>(v11.z);
            return v11.w;
        }
        case 7: // isect_quad_l3
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 936ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 952ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 968ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r11 = bitcast<unsigned int>(v2.z);
            R.r12 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 984ull * cap)[idx];
            R.r13 = bitcast<float>(v3.x);
            R.r14 = bitcast<unsigned int>(v3.y);
            R.r15 = bitcast<float>(v3.z);
            R.r16 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1000ull * cap)[idx];
            R.r17 = bitcast<float>(v4.x);
            R.r19 = bitcast<unsigned int>(v4.y);
            R.r22 = bitcast<float>(v4.z);
            R.r23 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1016ull * cap)[idx];
            R.r24 = bitcast<float>(v5.x);
            R.r25 = bitcast<float>(v5.y);
            R.r26 = bitcast<float>(v5.z);
            R.r27 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1032ull * cap)[idx];
            R.r28 = bitcast<float>(v6.x);
            R.r29 = bitcast<float>(v6.y);
            R.r30 = bitcast<float>(v6.z);
            R.r31 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1048ull * cap)[idx];
            R.r32 = bitcast<float>(v7.x);
            R.r33 = bitcast<float>(v7.y);
            R.r34 = bitcast<float>(v7.z);
            R.r35 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1064ull * cap)[idx];
            R.r36 = bitcast<float>(v8.x);
            R.r37 = bitcast<unsigned int>(v8.y);
            R.r38 = bitcast<unsigned int>(v8.z);
            R.r39 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 1080ull * cap)[idx];
            R.r40 = bitcast<unsigned int>(v9.x);
            R.r41 = bitcast<float>(v9.y);
            R.r42 = bitcast<float>(v9.z);
            R.r43 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 1096ull * cap)[idx];
            R.r44 = bitcast<float>(v10.x);
            R.r45 = bitcast<float>(v10.y);
            R.r46 = bitcast<float>(v10.z);
            R.r47 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 1112ull * cap)[idx];
            R.r62 = bitcast<float>(v11.x);
            R.r63 = bitcast<float>(v11.y);
            R.r64 = bitcast<float>(v11.z);
            return v11.w;
        }
        case 8: // isect_quad_l4
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1128ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1144ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1160ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1176ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1192ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1208ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1224ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1240ull * cap)[idx];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1256ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 1272ull * cap)[idx];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<float>(v9.y);
            R.r44 = bitcast<float>(v9.z);
            R.r45 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 1288ull * cap)[idx];
            R.r46 = bitcast<float>(v10.x);
            R.r47 = bitcast<float>(v10.y);
            R.r62 = bitcast<float>(v10.z);
            R.r63 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(base + 1304ull * cap)[idx];
            R.r64 = bitcast<float>(v11.x);
            return v11.y;
        }
        case 9: // isect_quad_l5
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1312ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1328ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1344ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1360ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1376ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1392ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1408ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1424ull * cap)[idx];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1440ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 1456ull * cap)[idx];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<float>(v9.y);
            R.r44 = bitcast<float>(v9.z);
            R.r45 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 1472ull * cap)[idx];
            R.r46 = bitcast<float>(v10.x);
            R.r47 = bitcast<float>(v10.y);
            R.r48 = bitcast<float>(v10.z);
            R.r49 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 1488ull * cap)[idx];
            R.r50 = bitcast<float>(v11.x);
            R.r55 = bitcast<float>(v11.y);
            R.r56 = bitcast<float>(v11.z);
            R.r57 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 1504ull * cap)[idx];
            R.r58 = bitcast<unsigned int>(v12.x);
            R.r62 = bitcast<float>(v12.y);
            R.r63 = bitcast<float>(v12.z);
            R.r64 = bitcast<float>(v12.w);
            const unsigned v13 = reinterpret_cast<const unsigned*>(base + 1520ull * cap)[idx];
            return v13;
        }
        case 10: // isect_quad_l6
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1528ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1544ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1560ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1576ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1592ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1608ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1624ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1640ull * cap)[idx];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1656ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 1672ull * cap)[idx];
            R.r45 = bitcast<float>(v9.x);
            R.r46 = bitcast<float>(v9.y);
            R.r47 = bitcast<float>(v9.z);
            R.r48 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 1688ull * cap)[idx];
            R.r49 = bitcast<float>(v10.x);
            R.r50 = bitcast<float>(v10.y);
            R.r51 = bitcast<float>(v10.z);
            R.r52 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 1704ull * cap)[idx];
            R.r53 = bitcast<float>(v11.x);
            R.r58 = bitcast<unsigned int>(v11.y);
            R.r62 = bitcast<float>(v11.z);
            R.r63 = bitcast<float>(v11.w);
            const uint2 v12 = reinterpret_cast<const uint2*>(base + 1720ull * cap)[idx];
            R.r64 = bitcast<float>(v12.x);
            return v12.y;
        }
        case 11: // isect_quad_l7
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1728ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1744ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1760ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1776ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1792ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1808ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1824ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1840ull * cap)[idx];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1856ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 1872ull * cap)[idx];
            R.r45 = bitcast<float>(v9.x);
            R.r46 = bitcast<float>(v9.y);
            R.r47 = bitcast<float>(v9.z);
            R.r62 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 1888ull * cap)[idx];
            R.r63 = bitcast<float>(v10.x);
            R.r64 = bitcast<float>(v10.y);
            return v10.z;
        }
        case 12: // isect_quad_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1904ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1920ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1936ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1952ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1968ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1984ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2000ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2016ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r54 = bitcast<unsigned int>(v7.y);
            R.r58 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2032ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            return v8.z;
        }
        case 13: // traverse_tetrahedron
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2048ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2064ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2080ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2096ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2112ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2128ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2144ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2160ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(base + 2176ull * cap)[idx];
            return v8;
        }
        case 14: // isect_triangle_mid1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2184ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2200ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2216ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2232ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2248ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2264ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2280ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2296ull * cap)[idx];
            R.r35 = bitcast<float>(v7.x);
            R.r36 = bitcast<float>(v7.y);
            R.r37 = bitcast<unsigned int>(v7.z);
            R.r38 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2312ull * cap)[idx];
            R.r39 = bitcast<float>(v8.x);
            R.r40 = bitcast<unsigned int>(v8.y);
            R.r41 = bitcast<float>(v8.z);
            R.r42 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 2328ull * cap)[idx];
            R.r43 = bitcast<float>(v9.x);
            R.r44 = bitcast<float>(v9.y);
            R.r45 = bitcast<float>(v9.z);
            R.r46 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 2344ull * cap)[idx];
            R.r47 = bitcast<float>(v10.x);
            R.r58 = bitcast<unsigned int>(v10.y);
            R.r62 = bitcast<float>(v10.z);
            R.r63 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(base + 2360ull * cap)[idx];
            R.r64 = bitcast<float>(v11.x);
            return v11.y;
        }
        case 15: // isect_triangle_mid2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2368ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2384ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2400ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2416ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2432ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2448ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2464ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2480ull * cap)[idx];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2496ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 2512ull * cap)[idx];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<float>(v9.y);
            R.r44 = bitcast<float>(v9.z);
            R.r58 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 2528ull * cap)[idx];
            R.r62 = bitcast<float>(v10.x);
            R.r63 = bitcast<float>(v10.y);
            R.r64 = bitcast<float>(v10.z);
            return v10.w;
        }
        case 16: // isect_triangle_mid3
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2544ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2560ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2576ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2592ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2608ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2624ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2640ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2656ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r42 = bitcast<float>(v7.y);
            R.r43 = bitcast<float>(v7.z);
            R.r44 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2672ull * cap)[idx];
            R.r45 = bitcast<float>(v8.x);
            R.r46 = bitcast<float>(v8.y);
            R.r47 = bitcast<float>(v8.z);
            R.r58 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 2688ull * cap)[idx];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            return v9.w;
        }
        case 17: // isect_triangle_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2704ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2720ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2736ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2752ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2768ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2784ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2800ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2816ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r54 = bitcast<unsigned int>(v7.y);
            R.r58 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2832ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            return v8.z;
        }
        case 18: // traverse_sphere
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2848ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2864ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2880ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2896ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2912ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2928ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2944ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2960ull * cap)[idx];
            R.r58 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(base + 2976ull * cap)[idx];
            return v8;
        }
        case 19: // traverse_solve_quadratic
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2984ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3000ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3016ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3032ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3048ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3064ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3080ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3096ull * cap)[idx];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3112ull * cap)[idx];
            R.r41 = bitcast<float>(v8.x);
            R.r58 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 3128ull * cap)[idx];
            R.r64 = bitcast<float>(v9.x);
            return v9.y;
        }
        case 20: // sq_head1
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
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3184ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3200ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3216ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3232ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3248ull * cap)[idx];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r40 = bitcast<unsigned int>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3264ull * cap)[idx];
            R.r58 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const unsigned v9 = reinterpret_cast<const unsigned*>(base + 3280ull * cap)[idx];
            return v9;
        }
        case 21: // sq_head2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3288ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3304ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3320ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3336ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3352ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3368ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3384ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3400ull * cap)[idx];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r40 = bitcast<unsigned int>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3416ull * cap)[idx];
            R.r54 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const unsigned v9 = reinterpret_cast<const unsigned*>(base + 3432ull * cap)[idx];
            return v9;
        }
        case 22: // sq_mid1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3440ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3456ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3472ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3488ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3504ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3520ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3536ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3552ull * cap)[idx];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3568ull * cap)[idx];
            R.r41 = bitcast<float>(v8.x);
            R.r58 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 3584ull * cap)[idx];
            R.r64 = bitcast<float>(v9.x);
            return v9.y;
        }
        case 23: // sq_mid2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3592ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3608ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3624ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3640ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3656ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3672ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3688ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r34 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3704ull * cap)[idx];
            R.r36 = bitcast<float>(v7.x);
            R.r37 = bitcast<unsigned int>(v7.y);
            R.r38 = bitcast<unsigned int>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3720ull * cap)[idx];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<float>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 3736ull * cap)[idx];
            R.r64 = bitcast<float>(v9.x);
            return v9.y;
        }
        case 24: // sq_mid
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3744ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3760ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3776ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3792ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3808ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3824ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3840ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r34 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3856ull * cap)[idx];
            R.r36 = bitcast<float>(v7.x);
            R.r37 = bitcast<unsigned int>(v7.y);
            R.r38 = bitcast<unsigned int>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3872ull * cap)[idx];
            R.r58 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const unsigned v9 = reinterpret_cast<const unsigned*>(base + 3888ull * cap)[idx];
            return v9;
        }
        case 25: // sq_tail
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3896ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3912ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3928ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3944ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3960ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3976ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3992ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r34 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4008ull * cap)[idx];
            R.r36 = bitcast<float>(v7.x);
            R.r37 = bitcast<unsigned int>(v7.y);
            R.r38 = bitcast<unsigned int>(v7.z);
            R.r58 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4024ull * cap)[idx];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            return v8.w;
        }
        case 26: // sq_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4040ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4056ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4072ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4088ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4104ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4120ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4136ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4152ull * cap)[idx];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r54 = bitcast<unsigned int>(v7.z);
            R.r58 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4168ull * cap)[idx];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            return v8.w;
        }
        case 27: // traverse_sphere_fin
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4184ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4200ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4216ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4232ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4248ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4264ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4280ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4296ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r54 = bitcast<unsigned int>(v7.y);
            R.r58 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4312ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            return v8.z;
        }
        case 28: // traverse_cylinder
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4328ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4344ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4360ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4376ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4392ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4408ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4424ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4440ull * cap)[idx];
            R.r58 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(base + 4456ull * cap)[idx];
            return v8;
        }
        case 29: // traverse_cylinder_fin
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4464ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4480ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4496ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4512ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4528ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4544ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4560ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4576ull * cap)[idx];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r54 = bitcast<unsigned int>(v7.z);
            R.r58 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4592ull * cap)[idx];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            return v8.w;
        }
        case 30: // traverse_disk
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4608ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4624ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4640ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4656ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4672ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4688ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4704ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4720ull * cap)[idx];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4736ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 4752ull * cap)[idx];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            return v9.w;
        }
        case 31: // isect_disk_rest
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4768ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4784ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4800ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4816ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4832ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4848ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4864ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4880ull * cap)[idx];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4896ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r58 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 4912ull * cap)[idx];
            R.r64 = bitcast<float>(v9.x);
            return v9.y;
        }
        case 32: // isect_disk_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4920ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4936ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4952ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4968ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4984ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5000ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5016ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 5032ull * cap)[idx];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r54 = bitcast<unsigned int>(v7.y);
            R.r58 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 5048ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            return v8.z;
        }
        case 33: // traverse_room_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5064ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5080ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5096ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5112ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5128ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5144ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5160ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 5176ull * cap)[idx];
            R.r58 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(base + 5192ull * cap)[idx];
            return v8;
        }
        case 34: // radiance
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5200ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5216ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5232ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5248ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5264ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5280ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5296ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 5312ull * cap)[idx];
            R.r58 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(base + 5328ull * cap)[idx];
            return v8;
        }
        case 35: // set_materials
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5336ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5352ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5368ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5384ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5400ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5416ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r31 = bitcast<unsigned int>(v5.y);
            R.r32 = bitcast<float>(v5.z);
            R.r36 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5432ull * cap)[idx];
            R.r37 = bitcast<unsigned int>(v6.x);
            R.r58 = bitcast<unsigned int>(v6.y);
            return v6.z;
        }
        case 36: // set_polygon_normal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5448ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5464ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5480ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5496ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5512ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5528ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5544ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r37 = bitcast<unsigned int>(v6.z);
            R.r58 = bitcast<unsigned int>(v6.w);
            const unsigned v7 = reinterpret_cast<const unsigned*>(base + 5560ull * cap)[idx];
            return v7;
        }
        case 37: // set_disk_normal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5568ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5584ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5600ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5616ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5632ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5648ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5664ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r37 = bitcast<unsigned int>(v6.z);
            R.r58 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 5680ull * cap)[idx];
            R.r59 = bitcast<float>(v7.x);
            R.r60 = bitcast<float>(v7.y);
            R.r61 = bitcast<float>(v7.z);
            return v7.w;
        }
        case 38: // compute_sphere_normal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5696ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5712ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5728ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5744ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5760ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5776ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5792ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 39: // compute_cylinder_normal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5808ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5824ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5840ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5856ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5872ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5888ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5904ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 40: // set_materials_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5920ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5936ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5952ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5968ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5984ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 6000ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 6016ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            R.r62 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 6032ull * cap)[idx];
            R.r63 = bitcast<float>(v7.x);
            R.r64 = bitcast<float>(v7.y);
            return v7.z;
        }
        case 41: // lambert_indirect
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 6048ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 6064ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r8 = bitcast<unsigned int>(v1.y);
            R.r9 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 6080ull * cap)[idx];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r16 = bitcast<float>(v2.z);
            R.r17 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 6096ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<unsigned int>(v3.y);
            R.r21 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 6112ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 6128ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 6144ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r58 = bitcast<unsigned int>(v6.y);
            R.r62 = bitcast<float>(v6.z);
            R.r63 = bitcast<float>(v6.w);
            const uint2 v7 = reinterpret_cast<const uint2*>(base + 6160ull * cap)[idx];
            R.r64 = bitcast<float>(v7.x);
            return v7.y;
        }
        case 42: // fin_sample
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 6168ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 6184ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 6200ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 6216ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 6232ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 6248ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 6264ull * cap)[idx];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            R.r62 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 6280ull * cap)[idx];
            R.r63 = bitcast<float>(v7.x);
            R.r64 = bitcast<float>(v7.y);
            return v7.z;
        }
        case 43: // fin_pixel
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 6296ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 6312ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r19 = bitcast<unsigned int>(v1.y);
            return v1.z;
        }
        default: return 0xffffffffu;
        }
    }

    // bytes of one queue entry's slots, the largest over the queues
    static constexpr unsigned kMaxStageRow = 224u;
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
        case 0: bytes = 2176u; break;
        case 1: bytes = 4096u; break;
        case 2: bytes = 2560u; break;
        case 3: bytes = 4096u; break;
        case 4: bytes = 4352u; break;
        case 5: bytes = 6400u; break;
        case 6: bytes = 6144u; break;
        case 7: bytes = 6144u; break;
        case 8: bytes = 5888u; break;
        case 9: bytes = 6784u; break;
        case 10: bytes = 6400u; break;
        case 11: bytes = 5632u; break;
        case 12: bytes = 4608u; break;
        case 13: bytes = 4224u; break;
        case 14: bytes = 5888u; break;
        case 15: bytes = 5632u; break;
        case 16: bytes = 5120u; break;
        case 17: bytes = 4608u; break;
        case 18: bytes = 4224u; break;
        case 19: bytes = 4864u; break;
        case 20: bytes = 4736u; break;
        case 21: bytes = 4736u; break;
        case 22: bytes = 4864u; break;
        case 23: bytes = 4864u; break;
        case 24: bytes = 4736u; break;
        case 25: bytes = 4608u; break;
        case 26: bytes = 4608u; break;
        case 27: bytes = 4608u; break;
        case 28: bytes = 4224u; break;
        case 29: bytes = 4608u; break;
        case 30: bytes = 5120u; break;
        case 31: bytes = 4864u; break;
        case 32: bytes = 4608u; break;
        case 33: bytes = 4224u; break;
        case 34: bytes = 4224u; break;
        case 35: bytes = 3584u; break;
        case 36: bytes = 3712u; break;
        case 37: bytes = 4096u; break;
        case 38: bytes = 3584u; break;
        case 39: bytes = 3584u; break;
        case 40: bytes = 4096u; break;
        case 41: bytes = 3840u; break;
        case 42: bytes = 4096u; break;
        case 43: bytes = 1024u; break;
        default: return false;
        }
        if((reinterpret_cast<unsigned long long>(base) | reinterpret_cast<unsigned long long>(stage)) & 15ull) return false;
        bulk_expect(mbar, bytes);
        switch(q)
        {
        case 0:
            bulk_copy(stage + 0u, base + 0ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 16ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 32ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 48ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 64ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 1:
            bulk_copy(stage + 0u, base + 72ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 88ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 2:
            bulk_copy(stage + 0u, base + 200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 3:
            bulk_copy(stage + 0u, base + 280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 4:
            bulk_copy(stage + 0u, base + 408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 472ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 520ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 536ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 5:
            bulk_copy(stage + 0u, base + 544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 736ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 6:
            bulk_copy(stage + 0u, base + 744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 7:
            bulk_copy(stage + 0u, base + 936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 968ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 1096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 1112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 8:
            bulk_copy(stage + 0u, base + 1128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1176ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1192ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1208ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1224ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 1288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 1304ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 9:
            bulk_copy(stage + 0u, base + 1312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 1472ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 1488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 1504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 1520ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 10:
            bulk_copy(stage + 0u, base + 1528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 1688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 1704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 1720ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 11:
            bulk_copy(stage + 0u, base + 1728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 1888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 12:
            bulk_copy(stage + 0u, base + 1904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1968ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 13:
            bulk_copy(stage + 0u, base + 2048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2176ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 14:
            bulk_copy(stage + 0u, base + 2184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 2328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 2344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 2360ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 15:
            bulk_copy(stage + 0u, base + 2368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 2512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 2528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 16:
            bulk_copy(stage + 0u, base + 2544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 2688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 17:
            bulk_copy(stage + 0u, base + 2704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2736ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2752ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2768ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2784ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2800ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2816ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2832ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 18:
            bulk_copy(stage + 0u, base + 2848ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2864ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2880ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2896ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2912ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2928ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2944ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2976ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 19:
            bulk_copy(stage + 0u, base + 2984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3128ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 20:
            bulk_copy(stage + 0u, base + 3136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3280ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 21:
            bulk_copy(stage + 0u, base + 3288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3304ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3320ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3432ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 22:
            bulk_copy(stage + 0u, base + 3440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3472ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3520ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3536ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3552ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3584ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 23:
            bulk_copy(stage + 0u, base + 3592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3736ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 24:
            bulk_copy(stage + 0u, base + 3744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3888ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 25:
            bulk_copy(stage + 0u, base + 3896ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3912ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3928ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3944ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4024ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 26:
            bulk_copy(stage + 0u, base + 4040ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 27:
            bulk_copy(stage + 0u, base + 4184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 28:
            bulk_copy(stage + 0u, base + 4328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4456ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 29:
            bulk_copy(stage + 0u, base + 4464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 30:
            bulk_copy(stage + 0u, base + 4608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4736ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 4752ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 31:
            bulk_copy(stage + 0u, base + 4768ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4784ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4800ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4816ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4832ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4848ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4864ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4880ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4896ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 4912ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 32:
            bulk_copy(stage + 0u, base + 4920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4968ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 5048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 33:
            bulk_copy(stage + 0u, base + 5064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5176ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 5192ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 34:
            bulk_copy(stage + 0u, base + 5200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 5328ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 35:
            bulk_copy(stage + 0u, base + 5336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 36:
            bulk_copy(stage + 0u, base + 5448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5560ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 37:
            bulk_copy(stage + 0u, base + 5568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5584ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5600ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5616ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5632ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5648ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5664ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5680ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 38:
            bulk_copy(stage + 0u, base + 5696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 39:
            bulk_copy(stage + 0u, base + 5808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 40:
            bulk_copy(stage + 0u, base + 5920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5968ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 6000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 6016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 6032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 41:
            bulk_copy(stage + 0u, base + 6048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 6064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 6080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 6096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 6112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 6128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 6144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 6160ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 42:
            bulk_copy(stage + 0u, base + 6168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 6184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 6200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 6216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 6232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 6248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 6264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 6280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 43:
            bulk_copy(stage + 0u, base + 6296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 6312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
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
            R.r22 = bitcast<float>(v0.y);
            R.r23 = bitcast<float>(v0.z);
            R.r24 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r25 = bitcast<float>(v1.x);
            R.r26 = bitcast<float>(v1.y);
            R.r27 = bitcast<float>(v1.z);
            R.r28 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r29 = bitcast<float>(v2.x);
            R.r30 = bitcast<float>(v2.y);
            R.r31 = bitcast<unsigned int>(v2.z);
            R.r32 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r58 = bitcast<unsigned int>(v3.x);
            R.r62 = bitcast<float>(v3.y);
            R.r63 = bitcast<float>(v3.z);
            R.r64 = bitcast<float>(v3.w);
            const unsigned v4 = reinterpret_cast<const unsigned*>(stage + 2048u)[lane];
            return v4;
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
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r58 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r62 = bitcast<float>(v7.x);
            R.r63 = bitcast<float>(v7.y);
            R.r64 = bitcast<float>(v7.z);
            return v7.w;
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
            R.r8 = bitcast<unsigned int>(v1.y);
            R.r9 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r16 = bitcast<float>(v2.z);
            R.r17 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r19 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<unsigned int>(v3.y);
            R.r21 = bitcast<unsigned int>(v3.z);
            R.r58 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r62 = bitcast<float>(v4.x);
            R.r63 = bitcast<float>(v4.y);
            R.r64 = bitcast<float>(v4.z);
            return v4.w;
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
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            R.r62 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r63 = bitcast<float>(v7.x);
            R.r64 = bitcast<float>(v7.y);
            return v7.z;
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
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r58 = bitcast<unsigned int>(v7.y);
            R.r62 = bitcast<float>(v7.z);
            R.r63 = bitcast<float>(v7.w);
            const uint2 v8 = reinterpret_cast<const uint2*>(stage + 4096u)[lane];
            R.r64 = bitcast<float>(v8.x);
            return v8.y;
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
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<float>(v9.y);
            R.r44 = bitcast<float>(v9.z);
            R.r45 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r46 = bitcast<float>(v10.x);
            R.r47 = bitcast<float>(v10.y);
            R.r55 = bitcast<float>(v10.z);
            R.r56 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r57 = bitcast<float>(v11.x);
            R.r58 = bitcast<unsigned int>(v11.y);
            R.r62 = bitcast<float>(v11.z);
            R.r63 = bitcast<float>(v11.w);
            const uint2 v12 = reinterpret_cast<const uint2*>(stage + 6144u)[lane];
            R.r64 = bitcast<float>(v12.x);
            return v12.y;
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
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r12 = bitcast<float>(v2.z);
            R.r13 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r14 = bitcast<unsigned int>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r16 = bitcast<float>(v3.z);
            R.r17 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<unsigned int>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<float>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<unsigned int>(v8.x);
            R.r38 = bitcast<unsigned int>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r41 = bitcast<float>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<float>(v9.z);
            R.r44 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r58 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r62 = bitcast<float>(v11.x);
            R.r63 = bitcast<float>(v11.y);
            R.r64 = bitcast<float>(v11.z);
            return v11.w;
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
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r11 = bitcast<unsigned int>(v2.z);
            R.r12 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r13 = bitcast<float>(v3.x);
            R.r14 = bitcast<unsigned int>(v3.y);
            R.r15 = bitcast<float>(v3.z);
            R.r16 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r17 = bitcast<float>(v4.x);
            R.r19 = bitcast<unsigned int>(v4.y);
            R.r22 = bitcast<float>(v4.z);
            R.r23 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r24 = bitcast<float>(v5.x);
            R.r25 = bitcast<float>(v5.y);
            R.r26 = bitcast<float>(v5.z);
            R.r27 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r28 = bitcast<float>(v6.x);
            R.r29 = bitcast<float>(v6.y);
            R.r30 = bitcast<float>(v6.z);
            R.r31 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r32 = bitcast<float>(v7.x);
            R.r33 = bitcast<float>(v7.y);
            R.r34 = bitcast<float>(v7.z);
            R.r35 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r36 = bitcast<float>(v8.x);
            R.r37 = bitcast<unsigned int>(v8.y);
            R.r38 = bitcast<unsigned int>(v8.z);
            R.r39 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r40 = bitcast<unsigned int>(v9.x);
            R.r41 = bitcast<float>(v9.y);
            R.r42 = bitcast<float>(v9.z);
            R.r43 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r44 = bitcast<float>(v10.x);
            R.r45 = bitcast<float>(v10.y);
            R.r46 = bitcast<float>(v10.z);
            R.r47 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r62 = bitcast<float>(v11.x);
            R.r63 = bitcast<float>(v11.y);
            R.r64 = bitcast<float>(v11.z);
            return v11.w;
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
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<float>(v9.y);
            R.r44 = bitcast<float>(v9.z);
            R.r45 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r46 = bitcast<float>(v10.x);
            R.r47 = bitcast<float>(v10.y);
            R.r62 = bitcast<float>(v10.z);
            R.r63 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(stage + 5632u)[lane];
            R.r64 = bitcast<float>(v11.x);
            return v11.y;
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
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<float>(v9.y);
            R.r44 = bitcast<float>(v9.z);
            R.r45 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r46 = bitcast<float>(v10.x);
            R.r47 = bitcast<float>(v10.y);
            R.r48 = bitcast<float>(v10.z);
            R.r49 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r50 = bitcast<float>(v11.x);
            R.r55 = bitcast<float>(v11.y);
            R.r56 = bitcast<float>(v11.z);
            R.r57 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r58 = bitcast<unsigned int>(v12.x);
            R.r62 = bitcast<float>(v12.y);
            R.r63 = bitcast<float>(v12.z);
            R.r64 = bitcast<float>(v12.w);
            const unsigned v13 = reinterpret_cast<const unsigned*>(stage + 6656u)[lane];
            return v13;
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
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r45 = bitcast<float>(v9.x);
            R.r46 = bitcast<float>(v9.y);
            R.r47 = bitcast<float>(v9.z);
            R.r48 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r49 = bitcast<float>(v10.x);
            R.r50 = bitcast<float>(v10.y);
            R.r51 = bitcast<float>(v10.z);
            R.r52 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r53 = bitcast<float>(v11.x);
            R.r58 = bitcast<unsigned int>(v11.y);
            R.r62 = bitcast<float>(v11.z);
            R.r63 = bitcast<float>(v11.w);
            const uint2 v12 = reinterpret_cast<const uint2*>(stage + 6144u)[lane];
            R.r64 = bitcast<float>(v12.x);
            return v12.y;
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
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r45 = bitcast<float>(v9.x);
            R.r46 = bitcast<float>(v9.y);
            R.r47 = bitcast<float>(v9.z);
            R.r62 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r63 = bitcast<float>(v10.x);
            R.r64 = bitcast<float>(v10.y);
            return v10.z;
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r54 = bitcast<unsigned int>(v7.y);
            R.r58 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            return v8.z;
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
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(stage + 4096u)[lane];
            return v8;
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r35 = bitcast<float>(v7.x);
            R.r36 = bitcast<float>(v7.y);
            R.r37 = bitcast<unsigned int>(v7.z);
            R.r38 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r39 = bitcast<float>(v8.x);
            R.r40 = bitcast<unsigned int>(v8.y);
            R.r41 = bitcast<float>(v8.z);
            R.r42 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r43 = bitcast<float>(v9.x);
            R.r44 = bitcast<float>(v9.y);
            R.r45 = bitcast<float>(v9.z);
            R.r46 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r47 = bitcast<float>(v10.x);
            R.r58 = bitcast<unsigned int>(v10.y);
            R.r62 = bitcast<float>(v10.z);
            R.r63 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(stage + 5632u)[lane];
            R.r64 = bitcast<float>(v11.x);
            return v11.y;
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
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<float>(v9.y);
            R.r44 = bitcast<float>(v9.z);
            R.r58 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r62 = bitcast<float>(v10.x);
            R.r63 = bitcast<float>(v10.y);
            R.r64 = bitcast<float>(v10.z);
            return v10.w;
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r42 = bitcast<float>(v7.y);
            R.r43 = bitcast<float>(v7.z);
            R.r44 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r45 = bitcast<float>(v8.x);
            R.r46 = bitcast<float>(v8.y);
            R.r47 = bitcast<float>(v8.z);
            R.r58 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            return v9.w;
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r54 = bitcast<unsigned int>(v7.y);
            R.r58 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            return v8.z;
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r58 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(stage + 4096u)[lane];
            return v8;
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<float>(v8.x);
            R.r58 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r64 = bitcast<float>(v9.x);
            return v9.y;
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r40 = bitcast<unsigned int>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r58 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const unsigned v9 = reinterpret_cast<const unsigned*>(stage + 4608u)[lane];
            return v9;
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
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r40 = bitcast<unsigned int>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r54 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const unsigned v9 = reinterpret_cast<const unsigned*>(stage + 4608u)[lane];
            return v9;
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
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<float>(v8.x);
            R.r58 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r64 = bitcast<float>(v9.x);
            return v9.y;
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
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r34 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r36 = bitcast<float>(v7.x);
            R.r37 = bitcast<unsigned int>(v7.y);
            R.r38 = bitcast<unsigned int>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<float>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r64 = bitcast<float>(v9.x);
            return v9.y;
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
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r34 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r36 = bitcast<float>(v7.x);
            R.r37 = bitcast<unsigned int>(v7.y);
            R.r38 = bitcast<unsigned int>(v7.z);
            R.r41 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r58 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const unsigned v9 = reinterpret_cast<const unsigned*>(stage + 4608u)[lane];
            return v9;
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
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r34 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r36 = bitcast<float>(v7.x);
            R.r37 = bitcast<unsigned int>(v7.y);
            R.r38 = bitcast<unsigned int>(v7.z);
            R.r58 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            return v8.w;
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r54 = bitcast<unsigned int>(v7.z);
            R.r58 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            return v8.w;
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r54 = bitcast<unsigned int>(v7.y);
            R.r58 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            return v8.z;
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
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r58 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(stage + 4096u)[lane];
            return v8;
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
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r34 = bitcast<float>(v6.z);
            R.r36 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r37 = bitcast<unsigned int>(v7.x);
            R.r38 = bitcast<unsigned int>(v7.y);
            R.r54 = bitcast<unsigned int>(v7.z);
            R.r58 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            return v8.w;
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
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            return v9.w;
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
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<unsigned int>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<float>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r38 = bitcast<unsigned int>(v8.x);
            R.r58 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r64 = bitcast<float>(v9.x);
            return v9.y;
        }
        case 32:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r38 = bitcast<unsigned int>(v7.x);
            R.r54 = bitcast<unsigned int>(v7.y);
            R.r58 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            return v8.z;
        }
        case 33:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r58 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(stage + 4096u)[lane];
            return v8;
        }
        case 34:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r36 = bitcast<float>(v6.z);
            R.r37 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r58 = bitcast<unsigned int>(v7.x);
            R.r62 = bitcast<float>(v7.y);
            R.r63 = bitcast<float>(v7.z);
            R.r64 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(stage + 4096u)[lane];
            return v8;
        }
        case 35:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r31 = bitcast<unsigned int>(v5.y);
            R.r32 = bitcast<float>(v5.z);
            R.r36 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r37 = bitcast<unsigned int>(v6.x);
            R.r58 = bitcast<unsigned int>(v6.y);
            return v6.z;
        }
        case 36:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r37 = bitcast<unsigned int>(v6.z);
            R.r58 = bitcast<unsigned int>(v6.w);
            const unsigned v7 = reinterpret_cast<const unsigned*>(stage + 3584u)[lane];
            return v7;
        }
        case 37:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r37 = bitcast<unsigned int>(v6.z);
            R.r58 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r59 = bitcast<float>(v7.x);
            R.r60 = bitcast<float>(v7.y);
            R.r61 = bitcast<float>(v7.z);
            return v7.w;
        }
        case 38:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 39:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 40:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            R.r62 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r63 = bitcast<float>(v7.x);
            R.r64 = bitcast<float>(v7.y);
            return v7.z;
        }
        case 41:
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
            R.r16 = bitcast<float>(v2.z);
            R.r17 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r19 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<unsigned int>(v3.y);
            R.r21 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r58 = bitcast<unsigned int>(v6.y);
            R.r62 = bitcast<float>(v6.z);
            R.r63 = bitcast<float>(v6.w);
            const uint2 v7 = reinterpret_cast<const uint2*>(stage + 3584u)[lane];
            R.r64 = bitcast<float>(v7.x);
            return v7.y;
        }
        case 42:
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
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r31 = bitcast<unsigned int>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r58 = bitcast<unsigned int>(v6.z);
            R.r62 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r63 = bitcast<float>(v7.x);
            R.r64 = bitcast<float>(v7.y);
            return v7.z;
        }
        case 43:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r19 = bitcast<unsigned int>(v1.y);
            return v1.z;
        }
        default: return 0xffffffffu;
        }
    }
};

const int kInTypes[] = {LOOM_B200_U32};
const int kOutTypes[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kInNames[] = {"ppp"};
const char* const kOutNames[] = {"L0", "L1", "L2", "rc", "ppp"};
const uint32_t kInstrs[] = {27, 296, 34, 10, 31, 11, 20, 3, 19, 10, 13, 22, 7, 28, 12, 15, 7, 7, 25, 3, 3, 3, 5, 11, 4, 3, 2, 4, 13, 15, 14, 16, 13, 2, 10, 31, 4, 19, 12, 12, 2, 70, 23, 5};
const uint32_t kLive[] = {64, 124, 76, 120, 132, 196, 188, 188, 180, 208, 196, 168, 136, 128, 180, 172, 156, 136, 128, 148, 144, 144, 148, 148, 144, 140, 140, 136, 128, 140, 156, 148, 136, 128, 128, 104, 112, 124, 108, 108, 120, 116, 120, 24};

const loom_b200_kernel_info kInfo = {
    "pt_const_40", "107b56955f2949d4", 1u, 5u, kInTypes, kOutTypes, kInNames, kOutNames,
    44u, 65u, 260u, 64u, kInstrs, kLive};

const uint32_t kQRegs0[] = {1u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 58u, 62u, 63u, 64u};
const int kQTypes0[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames0[] = {"ppp", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs0[] = {0ull, 0ull, 0ull, 0ull, 16ull, 16ull, 16ull, 16ull, 32ull, 32ull, 32ull, 32ull, 48ull, 48ull, 48ull, 48ull};
const unsigned kQSubs0[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths0[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs1[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 58u, 62u, 63u, 64u};
const int kQTypes1[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames1[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs1[] = {72ull, 72ull, 72ull, 72ull, 88ull, 88ull, 88ull, 88ull, 104ull, 104ull, 104ull, 104ull, 120ull, 120ull, 120ull, 120ull, 136ull, 136ull, 136ull, 136ull, 152ull, 152ull, 152ull, 152ull, 168ull, 168ull, 168ull, 168ull, 184ull, 184ull, 184ull};
const unsigned kQSubs1[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths1[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs2[] = {1u, 2u, 3u, 4u, 5u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 21u, 58u, 62u, 63u, 64u};
const int kQTypes2[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames2[] = {"ppp", "L0", "L1", "L2", "rc", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "u1", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs2[] = {200ull, 200ull, 200ull, 200ull, 216ull, 216ull, 216ull, 216ull, 232ull, 232ull, 232ull, 232ull, 248ull, 248ull, 248ull, 248ull, 264ull, 264ull, 264ull};
const unsigned kQSubs2[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths2[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs3[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 58u, 62u, 63u, 64u};
const int kQTypes3[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames3[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs3[] = {280ull, 280ull, 280ull, 280ull, 296ull, 296ull, 296ull, 296ull, 312ull, 312ull, 312ull, 312ull, 328ull, 328ull, 328ull, 328ull, 344ull, 344ull, 344ull, 344ull, 360ull, 360ull, 360ull, 360ull, 376ull, 376ull, 376ull, 376ull, 392ull, 392ull};
const unsigned kQSubs3[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths3[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs4[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 38u, 58u, 62u, 63u, 64u};
const int kQTypes4[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames4[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs4[] = {408ull, 408ull, 408ull, 408ull, 424ull, 424ull, 424ull, 424ull, 440ull, 440ull, 440ull, 440ull, 456ull, 456ull, 456ull, 456ull, 472ull, 472ull, 472ull, 472ull, 488ull, 488ull, 488ull, 488ull, 504ull, 504ull, 504ull, 504ull, 520ull, 520ull, 520ull, 520ull, 536ull};
const unsigned kQSubs4[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths4[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs5[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 55u, 56u, 57u, 58u, 62u, 63u, 64u};
const int kQTypes5[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames5[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "vr60", "vr61", "vr62", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs5[] = {544ull, 544ull, 544ull, 544ull, 560ull, 560ull, 560ull, 560ull, 576ull, 576ull, 576ull, 576ull, 592ull, 592ull, 592ull, 592ull, 608ull, 608ull, 608ull, 608ull, 624ull, 624ull, 624ull, 624ull, 640ull, 640ull, 640ull, 640ull, 656ull, 656ull, 656ull, 656ull, 672ull, 672ull, 672ull, 672ull, 688ull, 688ull, 688ull, 688ull, 704ull, 704ull, 704ull, 704ull, 720ull, 720ull, 720ull, 720ull, 736ull};
const unsigned kQSubs5[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths5[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs6[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 10u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 58u, 62u, 63u, 64u};
const int kQTypes6[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames6[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "tmp1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs6[] = {744ull, 744ull, 744ull, 744ull, 760ull, 760ull, 760ull, 760ull, 776ull, 776ull, 776ull, 776ull, 792ull, 792ull, 792ull, 792ull, 808ull, 808ull, 808ull, 808ull, 824ull, 824ull, 824ull, 824ull, 840ull, 840ull, 840ull, 840ull, 856ull, 856ull, 856ull, 856ull, 872ull, 872ull, 872ull, 872ull, 888ull, 888ull, 888ull, 888ull, 904ull, 904ull, 904ull, 904ull, 920ull, 920ull, 920ull};
const unsigned kQSubs6[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths6[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs7[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 62u, 63u, 64u};
const int kQTypes7[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames7[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "tmp1", "tmp2", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "n0", "n1", "n2"};
const unsigned long long kQOffs7[] = {936ull, 936ull, 936ull, 936ull, 952ull, 952ull, 952ull, 952ull, 968ull, 968ull, 968ull, 968ull, 984ull, 984ull, 984ull, 984ull, 1000ull, 1000ull, 1000ull, 1000ull, 1016ull, 1016ull, 1016ull, 1016ull, 1032ull, 1032ull, 1032ull, 1032ull, 1048ull, 1048ull, 1048ull, 1048ull, 1064ull, 1064ull, 1064ull, 1064ull, 1080ull, 1080ull, 1080ull, 1080ull, 1096ull, 1096ull, 1096ull, 1096ull, 1112ull, 1112ull, 1112ull};
const unsigned kQSubs7[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths7[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs8[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 62u, 63u, 64u};
const int kQTypes8[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames8[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "n0", "n1", "n2"};
const unsigned long long kQOffs8[] = {1128ull, 1128ull, 1128ull, 1128ull, 1144ull, 1144ull, 1144ull, 1144ull, 1160ull, 1160ull, 1160ull, 1160ull, 1176ull, 1176ull, 1176ull, 1176ull, 1192ull, 1192ull, 1192ull, 1192ull, 1208ull, 1208ull, 1208ull, 1208ull, 1224ull, 1224ull, 1224ull, 1224ull, 1240ull, 1240ull, 1240ull, 1240ull, 1256ull, 1256ull, 1256ull, 1256ull, 1272ull, 1272ull, 1272ull, 1272ull, 1288ull, 1288ull, 1288ull, 1288ull, 1304ull};
const unsigned kQSubs8[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths8[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs9[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 48u, 49u, 50u, 55u, 56u, 57u, 58u, 62u, 63u, 64u};
const int kQTypes9[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames9[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "vr40", "vr41", "vr42", "vr60", "vr61", "vr62", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs9[] = {1312ull, 1312ull, 1312ull, 1312ull, 1328ull, 1328ull, 1328ull, 1328ull, 1344ull, 1344ull, 1344ull, 1344ull, 1360ull, 1360ull, 1360ull, 1360ull, 1376ull, 1376ull, 1376ull, 1376ull, 1392ull, 1392ull, 1392ull, 1392ull, 1408ull, 1408ull, 1408ull, 1408ull, 1424ull, 1424ull, 1424ull, 1424ull, 1440ull, 1440ull, 1440ull, 1440ull, 1456ull, 1456ull, 1456ull, 1456ull, 1472ull, 1472ull, 1472ull, 1472ull, 1488ull, 1488ull, 1488ull, 1488ull, 1504ull, 1504ull, 1504ull, 1504ull};
const unsigned kQSubs9[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths9[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs10[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 45u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 53u, 58u, 62u, 63u, 64u};
const int kQTypes10[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames10[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr30", "vr31", "vr32", "vr40", "vr41", "vr42", "vr50", "vr51", "vr52", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs10[] = {1528ull, 1528ull, 1528ull, 1528ull, 1544ull, 1544ull, 1544ull, 1544ull, 1560ull, 1560ull, 1560ull, 1560ull, 1576ull, 1576ull, 1576ull, 1576ull, 1592ull, 1592ull, 1592ull, 1592ull, 1608ull, 1608ull, 1608ull, 1608ull, 1624ull, 1624ull, 1624ull, 1624ull, 1640ull, 1640ull, 1640ull, 1640ull, 1656ull, 1656ull, 1656ull, 1656ull, 1672ull, 1672ull, 1672ull, 1672ull, 1688ull, 1688ull, 1688ull, 1688ull, 1704ull, 1704ull, 1704ull, 1704ull, 1720ull};
const unsigned kQSubs10[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths10[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs11[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 45u, 46u, 47u, 62u, 63u, 64u};
const int kQTypes11[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames11[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr30", "vr31", "vr32", "n0", "n1", "n2"};
const unsigned long long kQOffs11[] = {1728ull, 1728ull, 1728ull, 1728ull, 1744ull, 1744ull, 1744ull, 1744ull, 1760ull, 1760ull, 1760ull, 1760ull, 1776ull, 1776ull, 1776ull, 1776ull, 1792ull, 1792ull, 1792ull, 1792ull, 1808ull, 1808ull, 1808ull, 1808ull, 1824ull, 1824ull, 1824ull, 1824ull, 1840ull, 1840ull, 1840ull, 1840ull, 1856ull, 1856ull, 1856ull, 1856ull, 1872ull, 1872ull, 1872ull, 1872ull, 1888ull, 1888ull};
const unsigned kQSubs11[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths11[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs12[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 38u, 54u, 58u, 62u, 63u, 64u};
const int kQTypes12[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames12[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "hit", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs12[] = {1904ull, 1904ull, 1904ull, 1904ull, 1920ull, 1920ull, 1920ull, 1920ull, 1936ull, 1936ull, 1936ull, 1936ull, 1952ull, 1952ull, 1952ull, 1952ull, 1968ull, 1968ull, 1968ull, 1968ull, 1984ull, 1984ull, 1984ull, 1984ull, 2000ull, 2000ull, 2000ull, 2000ull, 2016ull, 2016ull, 2016ull, 2016ull, 2032ull, 2032ull};
const unsigned kQSubs12[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths12[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs13[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 38u, 62u, 63u, 64u};
const int kQTypes13[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames13[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "n0", "n1", "n2"};
const unsigned long long kQOffs13[] = {2048ull, 2048ull, 2048ull, 2048ull, 2064ull, 2064ull, 2064ull, 2064ull, 2080ull, 2080ull, 2080ull, 2080ull, 2096ull, 2096ull, 2096ull, 2096ull, 2112ull, 2112ull, 2112ull, 2112ull, 2128ull, 2128ull, 2128ull, 2128ull, 2144ull, 2144ull, 2144ull, 2144ull, 2160ull, 2160ull, 2160ull, 2160ull};
const unsigned kQSubs13[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths13[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs14[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 58u, 62u, 63u, 64u};
const int kQTypes14[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames14[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs14[] = {2184ull, 2184ull, 2184ull, 2184ull, 2200ull, 2200ull, 2200ull, 2200ull, 2216ull, 2216ull, 2216ull, 2216ull, 2232ull, 2232ull, 2232ull, 2232ull, 2248ull, 2248ull, 2248ull, 2248ull, 2264ull, 2264ull, 2264ull, 2264ull, 2280ull, 2280ull, 2280ull, 2280ull, 2296ull, 2296ull, 2296ull, 2296ull, 2312ull, 2312ull, 2312ull, 2312ull, 2328ull, 2328ull, 2328ull, 2328ull, 2344ull, 2344ull, 2344ull, 2344ull, 2360ull};
const unsigned kQSubs14[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths14[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs15[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 58u, 62u, 63u, 64u};
const int kQTypes15[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames15[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs15[] = {2368ull, 2368ull, 2368ull, 2368ull, 2384ull, 2384ull, 2384ull, 2384ull, 2400ull, 2400ull, 2400ull, 2400ull, 2416ull, 2416ull, 2416ull, 2416ull, 2432ull, 2432ull, 2432ull, 2432ull, 2448ull, 2448ull, 2448ull, 2448ull, 2464ull, 2464ull, 2464ull, 2464ull, 2480ull, 2480ull, 2480ull, 2480ull, 2496ull, 2496ull, 2496ull, 2496ull, 2512ull, 2512ull, 2512ull, 2512ull, 2528ull, 2528ull, 2528ull};
const unsigned kQSubs15[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths15[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs16[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 38u, 42u, 43u, 44u, 45u, 46u, 47u, 58u, 62u, 63u, 64u};
const int kQTypes16[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames16[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs16[] = {2544ull, 2544ull, 2544ull, 2544ull, 2560ull, 2560ull, 2560ull, 2560ull, 2576ull, 2576ull, 2576ull, 2576ull, 2592ull, 2592ull, 2592ull, 2592ull, 2608ull, 2608ull, 2608ull, 2608ull, 2624ull, 2624ull, 2624ull, 2624ull, 2640ull, 2640ull, 2640ull, 2640ull, 2656ull, 2656ull, 2656ull, 2656ull, 2672ull, 2672ull, 2672ull, 2672ull, 2688ull, 2688ull, 2688ull};
const unsigned kQSubs16[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths16[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs17[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 38u, 54u, 58u, 62u, 63u, 64u};
const int kQTypes17[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames17[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "hit", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs17[] = {2704ull, 2704ull, 2704ull, 2704ull, 2720ull, 2720ull, 2720ull, 2720ull, 2736ull, 2736ull, 2736ull, 2736ull, 2752ull, 2752ull, 2752ull, 2752ull, 2768ull, 2768ull, 2768ull, 2768ull, 2784ull, 2784ull, 2784ull, 2784ull, 2800ull, 2800ull, 2800ull, 2800ull, 2816ull, 2816ull, 2816ull, 2816ull, 2832ull, 2832ull};
const unsigned kQSubs17[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths17[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs18[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 58u, 62u, 63u, 64u};
const int kQTypes18[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames18[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs18[] = {2848ull, 2848ull, 2848ull, 2848ull, 2864ull, 2864ull, 2864ull, 2864ull, 2880ull, 2880ull, 2880ull, 2880ull, 2896ull, 2896ull, 2896ull, 2896ull, 2912ull, 2912ull, 2912ull, 2912ull, 2928ull, 2928ull, 2928ull, 2928ull, 2944ull, 2944ull, 2944ull, 2944ull, 2960ull, 2960ull, 2960ull, 2960ull};
const unsigned kQSubs18[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths18[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs19[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 34u, 36u, 37u, 38u, 39u, 40u, 41u, 58u, 62u, 63u, 64u};
const int kQTypes19[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames19[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs19[] = {2984ull, 2984ull, 2984ull, 2984ull, 3000ull, 3000ull, 3000ull, 3000ull, 3016ull, 3016ull, 3016ull, 3016ull, 3032ull, 3032ull, 3032ull, 3032ull, 3048ull, 3048ull, 3048ull, 3048ull, 3064ull, 3064ull, 3064ull, 3064ull, 3080ull, 3080ull, 3080ull, 3080ull, 3096ull, 3096ull, 3096ull, 3096ull, 3112ull, 3112ull, 3112ull, 3112ull, 3128ull};
const unsigned kQSubs19[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths19[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs20[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 34u, 36u, 37u, 38u, 40u, 41u, 58u, 62u, 63u, 64u};
const int kQTypes20[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames20[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr11", "vr12", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs20[] = {3136ull, 3136ull, 3136ull, 3136ull, 3152ull, 3152ull, 3152ull, 3152ull, 3168ull, 3168ull, 3168ull, 3168ull, 3184ull, 3184ull, 3184ull, 3184ull, 3200ull, 3200ull, 3200ull, 3200ull, 3216ull, 3216ull, 3216ull, 3216ull, 3232ull, 3232ull, 3232ull, 3232ull, 3248ull, 3248ull, 3248ull, 3248ull, 3264ull, 3264ull, 3264ull, 3264ull};
const unsigned kQSubs20[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths20[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs21[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 34u, 36u, 37u, 38u, 40u, 41u, 54u, 62u, 63u, 64u};
const int kQTypes21[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames21[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr11", "vr12", "hit", "n0", "n1", "n2"};
const unsigned long long kQOffs21[] = {3288ull, 3288ull, 3288ull, 3288ull, 3304ull, 3304ull, 3304ull, 3304ull, 3320ull, 3320ull, 3320ull, 3320ull, 3336ull, 3336ull, 3336ull, 3336ull, 3352ull, 3352ull, 3352ull, 3352ull, 3368ull, 3368ull, 3368ull, 3368ull, 3384ull, 3384ull, 3384ull, 3384ull, 3400ull, 3400ull, 3400ull, 3400ull, 3416ull, 3416ull, 3416ull, 3416ull};
const unsigned kQSubs21[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths21[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs22[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 34u, 36u, 37u, 38u, 39u, 40u, 41u, 58u, 62u, 63u, 64u};
const int kQTypes22[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames22[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs22[] = {3440ull, 3440ull, 3440ull, 3440ull, 3456ull, 3456ull, 3456ull, 3456ull, 3472ull, 3472ull, 3472ull, 3472ull, 3488ull, 3488ull, 3488ull, 3488ull, 3504ull, 3504ull, 3504ull, 3504ull, 3520ull, 3520ull, 3520ull, 3520ull, 3536ull, 3536ull, 3536ull, 3536ull, 3552ull, 3552ull, 3552ull, 3552ull, 3568ull, 3568ull, 3568ull, 3568ull, 3584ull};
const unsigned kQSubs22[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths22[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs23[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 34u, 36u, 37u, 38u, 39u, 40u, 41u, 62u, 63u, 64u};
const int kQTypes23[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames23[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "n0", "n1", "n2"};
const unsigned long long kQOffs23[] = {3592ull, 3592ull, 3592ull, 3592ull, 3608ull, 3608ull, 3608ull, 3608ull, 3624ull, 3624ull, 3624ull, 3624ull, 3640ull, 3640ull, 3640ull, 3640ull, 3656ull, 3656ull, 3656ull, 3656ull, 3672ull, 3672ull, 3672ull, 3672ull, 3688ull, 3688ull, 3688ull, 3688ull, 3704ull, 3704ull, 3704ull, 3704ull, 3720ull, 3720ull, 3720ull, 3720ull, 3736ull};
const unsigned kQSubs23[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths23[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs24[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 34u, 36u, 37u, 38u, 41u, 58u, 62u, 63u, 64u};
const int kQTypes24[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames24[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr12", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs24[] = {3744ull, 3744ull, 3744ull, 3744ull, 3760ull, 3760ull, 3760ull, 3760ull, 3776ull, 3776ull, 3776ull, 3776ull, 3792ull, 3792ull, 3792ull, 3792ull, 3808ull, 3808ull, 3808ull, 3808ull, 3824ull, 3824ull, 3824ull, 3824ull, 3840ull, 3840ull, 3840ull, 3840ull, 3856ull, 3856ull, 3856ull, 3856ull, 3872ull, 3872ull, 3872ull, 3872ull};
const unsigned kQSubs24[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths24[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs25[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 34u, 36u, 37u, 38u, 58u, 62u, 63u, 64u};
const int kQTypes25[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames25[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs25[] = {3896ull, 3896ull, 3896ull, 3896ull, 3912ull, 3912ull, 3912ull, 3912ull, 3928ull, 3928ull, 3928ull, 3928ull, 3944ull, 3944ull, 3944ull, 3944ull, 3960ull, 3960ull, 3960ull, 3960ull, 3976ull, 3976ull, 3976ull, 3976ull, 3992ull, 3992ull, 3992ull, 3992ull, 4008ull, 4008ull, 4008ull, 4008ull, 4024ull, 4024ull, 4024ull};
const unsigned kQSubs25[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths25[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs26[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 34u, 36u, 37u, 38u, 54u, 58u, 62u, 63u, 64u};
const int kQTypes26[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames26[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "hit", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs26[] = {4040ull, 4040ull, 4040ull, 4040ull, 4056ull, 4056ull, 4056ull, 4056ull, 4072ull, 4072ull, 4072ull, 4072ull, 4088ull, 4088ull, 4088ull, 4088ull, 4104ull, 4104ull, 4104ull, 4104ull, 4120ull, 4120ull, 4120ull, 4120ull, 4136ull, 4136ull, 4136ull, 4136ull, 4152ull, 4152ull, 4152ull, 4152ull, 4168ull, 4168ull, 4168ull};
const unsigned kQSubs26[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths26[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs27[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 38u, 54u, 58u, 62u, 63u, 64u};
const int kQTypes27[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames27[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "hit", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs27[] = {4184ull, 4184ull, 4184ull, 4184ull, 4200ull, 4200ull, 4200ull, 4200ull, 4216ull, 4216ull, 4216ull, 4216ull, 4232ull, 4232ull, 4232ull, 4232ull, 4248ull, 4248ull, 4248ull, 4248ull, 4264ull, 4264ull, 4264ull, 4264ull, 4280ull, 4280ull, 4280ull, 4280ull, 4296ull, 4296ull, 4296ull, 4296ull, 4312ull, 4312ull};
const unsigned kQSubs27[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths27[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs28[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 58u, 62u, 63u, 64u};
const int kQTypes28[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames28[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs28[] = {4328ull, 4328ull, 4328ull, 4328ull, 4344ull, 4344ull, 4344ull, 4344ull, 4360ull, 4360ull, 4360ull, 4360ull, 4376ull, 4376ull, 4376ull, 4376ull, 4392ull, 4392ull, 4392ull, 4392ull, 4408ull, 4408ull, 4408ull, 4408ull, 4424ull, 4424ull, 4424ull, 4424ull, 4440ull, 4440ull, 4440ull, 4440ull};
const unsigned kQSubs28[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths28[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs29[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 34u, 36u, 37u, 38u, 54u, 58u, 62u, 63u, 64u};
const int kQTypes29[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames29[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "hit", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs29[] = {4464ull, 4464ull, 4464ull, 4464ull, 4480ull, 4480ull, 4480ull, 4480ull, 4496ull, 4496ull, 4496ull, 4496ull, 4512ull, 4512ull, 4512ull, 4512ull, 4528ull, 4528ull, 4528ull, 4528ull, 4544ull, 4544ull, 4544ull, 4544ull, 4560ull, 4560ull, 4560ull, 4560ull, 4576ull, 4576ull, 4576ull, 4576ull, 4592ull, 4592ull, 4592ull};
const unsigned kQSubs29[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths29[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs30[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 62u, 63u, 64u};
const int kQTypes30[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames30[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "n0", "n1", "n2"};
const unsigned long long kQOffs30[] = {4608ull, 4608ull, 4608ull, 4608ull, 4624ull, 4624ull, 4624ull, 4624ull, 4640ull, 4640ull, 4640ull, 4640ull, 4656ull, 4656ull, 4656ull, 4656ull, 4672ull, 4672ull, 4672ull, 4672ull, 4688ull, 4688ull, 4688ull, 4688ull, 4704ull, 4704ull, 4704ull, 4704ull, 4720ull, 4720ull, 4720ull, 4720ull, 4736ull, 4736ull, 4736ull, 4736ull, 4752ull, 4752ull, 4752ull};
const unsigned kQSubs30[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths30[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs31[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 58u, 62u, 63u, 64u};
const int kQTypes31[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames31[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs31[] = {4768ull, 4768ull, 4768ull, 4768ull, 4784ull, 4784ull, 4784ull, 4784ull, 4800ull, 4800ull, 4800ull, 4800ull, 4816ull, 4816ull, 4816ull, 4816ull, 4832ull, 4832ull, 4832ull, 4832ull, 4848ull, 4848ull, 4848ull, 4848ull, 4864ull, 4864ull, 4864ull, 4864ull, 4880ull, 4880ull, 4880ull, 4880ull, 4896ull, 4896ull, 4896ull, 4896ull, 4912ull};
const unsigned kQSubs31[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths31[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs32[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 38u, 54u, 58u, 62u, 63u, 64u};
const int kQTypes32[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames32[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "hit", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs32[] = {4920ull, 4920ull, 4920ull, 4920ull, 4936ull, 4936ull, 4936ull, 4936ull, 4952ull, 4952ull, 4952ull, 4952ull, 4968ull, 4968ull, 4968ull, 4968ull, 4984ull, 4984ull, 4984ull, 4984ull, 5000ull, 5000ull, 5000ull, 5000ull, 5016ull, 5016ull, 5016ull, 5016ull, 5032ull, 5032ull, 5032ull, 5032ull, 5048ull, 5048ull};
const unsigned kQSubs32[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths32[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs33[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 58u, 62u, 63u, 64u};
const int kQTypes33[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames33[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs33[] = {5064ull, 5064ull, 5064ull, 5064ull, 5080ull, 5080ull, 5080ull, 5080ull, 5096ull, 5096ull, 5096ull, 5096ull, 5112ull, 5112ull, 5112ull, 5112ull, 5128ull, 5128ull, 5128ull, 5128ull, 5144ull, 5144ull, 5144ull, 5144ull, 5160ull, 5160ull, 5160ull, 5160ull, 5176ull, 5176ull, 5176ull, 5176ull};
const unsigned kQSubs33[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths33[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs34[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 36u, 37u, 58u, 62u, 63u, 64u};
const int kQTypes34[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames34[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs34[] = {5200ull, 5200ull, 5200ull, 5200ull, 5216ull, 5216ull, 5216ull, 5216ull, 5232ull, 5232ull, 5232ull, 5232ull, 5248ull, 5248ull, 5248ull, 5248ull, 5264ull, 5264ull, 5264ull, 5264ull, 5280ull, 5280ull, 5280ull, 5280ull, 5296ull, 5296ull, 5296ull, 5296ull, 5312ull, 5312ull, 5312ull, 5312ull};
const unsigned kQSubs34[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths34[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs35[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 31u, 32u, 36u, 37u, 58u};
const int kQTypes35[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames35[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "depth", "d2", "t", "pid", "ct"};
const unsigned long long kQOffs35[] = {5336ull, 5336ull, 5336ull, 5336ull, 5352ull, 5352ull, 5352ull, 5352ull, 5368ull, 5368ull, 5368ull, 5368ull, 5384ull, 5384ull, 5384ull, 5384ull, 5400ull, 5400ull, 5400ull, 5400ull, 5416ull, 5416ull, 5416ull, 5416ull, 5432ull, 5432ull};
const unsigned kQSubs35[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths35[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs36[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 37u, 58u};
const int kQTypes36[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames36[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "pid", "ct"};
const unsigned long long kQOffs36[] = {5448ull, 5448ull, 5448ull, 5448ull, 5464ull, 5464ull, 5464ull, 5464ull, 5480ull, 5480ull, 5480ull, 5480ull, 5496ull, 5496ull, 5496ull, 5496ull, 5512ull, 5512ull, 5512ull, 5512ull, 5528ull, 5528ull, 5528ull, 5528ull, 5544ull, 5544ull, 5544ull, 5544ull};
const unsigned kQSubs36[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths36[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs37[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 37u, 58u, 59u, 60u, 61u};
const int kQTypes37[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames37[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "pid", "ct", "t0", "t1", "t2"};
const unsigned long long kQOffs37[] = {5568ull, 5568ull, 5568ull, 5568ull, 5584ull, 5584ull, 5584ull, 5584ull, 5600ull, 5600ull, 5600ull, 5600ull, 5616ull, 5616ull, 5616ull, 5616ull, 5632ull, 5632ull, 5632ull, 5632ull, 5648ull, 5648ull, 5648ull, 5648ull, 5664ull, 5664ull, 5664ull, 5664ull, 5680ull, 5680ull, 5680ull};
const unsigned kQSubs37[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths37[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs38[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 58u};
const int kQTypes38[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames38[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "ct"};
const unsigned long long kQOffs38[] = {5696ull, 5696ull, 5696ull, 5696ull, 5712ull, 5712ull, 5712ull, 5712ull, 5728ull, 5728ull, 5728ull, 5728ull, 5744ull, 5744ull, 5744ull, 5744ull, 5760ull, 5760ull, 5760ull, 5760ull, 5776ull, 5776ull, 5776ull, 5776ull, 5792ull, 5792ull, 5792ull};
const unsigned kQSubs38[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths38[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs39[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 58u};
const int kQTypes39[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames39[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "ct"};
const unsigned long long kQOffs39[] = {5808ull, 5808ull, 5808ull, 5808ull, 5824ull, 5824ull, 5824ull, 5824ull, 5840ull, 5840ull, 5840ull, 5840ull, 5856ull, 5856ull, 5856ull, 5856ull, 5872ull, 5872ull, 5872ull, 5872ull, 5888ull, 5888ull, 5888ull, 5888ull, 5904ull, 5904ull, 5904ull};
const unsigned kQSubs39[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths39[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs40[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 58u, 62u, 63u, 64u};
const int kQTypes40[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames40[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs40[] = {5920ull, 5920ull, 5920ull, 5920ull, 5936ull, 5936ull, 5936ull, 5936ull, 5952ull, 5952ull, 5952ull, 5952ull, 5968ull, 5968ull, 5968ull, 5968ull, 5984ull, 5984ull, 5984ull, 5984ull, 6000ull, 6000ull, 6000ull, 6000ull, 6016ull, 6016ull, 6016ull, 6016ull, 6032ull, 6032ull};
const unsigned kQSubs40[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths40[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs41[] = {1u, 2u, 3u, 4u, 5u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 21u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 58u, 62u, 63u, 64u};
const int kQTypes41[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames41[] = {"ppp", "L0", "L1", "L2", "rc", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "u1", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs41[] = {6048ull, 6048ull, 6048ull, 6048ull, 6064ull, 6064ull, 6064ull, 6064ull, 6080ull, 6080ull, 6080ull, 6080ull, 6096ull, 6096ull, 6096ull, 6096ull, 6112ull, 6112ull, 6112ull, 6112ull, 6128ull, 6128ull, 6128ull, 6128ull, 6144ull, 6144ull, 6144ull, 6144ull, 6160ull};
const unsigned kQSubs41[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths41[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs42[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 58u, 62u, 63u, 64u};
const int kQTypes42[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames42[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "PL0", "PL1", "PL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "n0", "n1", "n2"};
const unsigned long long kQOffs42[] = {6168ull, 6168ull, 6168ull, 6168ull, 6184ull, 6184ull, 6184ull, 6184ull, 6200ull, 6200ull, 6200ull, 6200ull, 6216ull, 6216ull, 6216ull, 6216ull, 6232ull, 6232ull, 6232ull, 6232ull, 6248ull, 6248ull, 6248ull, 6248ull, 6264ull, 6264ull, 6264ull, 6264ull, 6280ull, 6280ull};
const unsigned kQSubs42[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths42[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs43[] = {1u, 2u, 3u, 4u, 5u, 19u};
const int kQTypes43[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames43[] = {"ppp", "L0", "L1", "L2", "rc", "ns"};
const unsigned long long kQOffs43[] = {6296ull, 6296ull, 6296ull, 6296ull, 6312ull, 6312ull};
const unsigned kQSubs43[] = {0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths43[] = {16u, 16u, 16u, 16u, 16u, 16u};
const loom_b200_queue_layout kQueues[] = {
    {0u, -1, 16u, kQRegs0, kQTypes0, kQNames0},
    {1u, -1, 31u, kQRegs1, kQTypes1, kQNames1},
    {2u, -1, 19u, kQRegs2, kQTypes2, kQNames2},
    {3u, -1, 30u, kQRegs3, kQTypes3, kQNames3},
    {4u, -1, 33u, kQRegs4, kQTypes4, kQNames4},
    {5u, -1, 49u, kQRegs5, kQTypes5, kQNames5},
    {6u, -1, 47u, kQRegs6, kQTypes6, kQNames6},
    {7u, -1, 47u, kQRegs7, kQTypes7, kQNames7},
    {8u, -1, 45u, kQRegs8, kQTypes8, kQNames8},
    {9u, -1, 52u, kQRegs9, kQTypes9, kQNames9},
    {10u, -1, 49u, kQRegs10, kQTypes10, kQNames10},
    {11u, -1, 42u, kQRegs11, kQTypes11, kQNames11},
    {12u, -1, 34u, kQRegs12, kQTypes12, kQNames12},
    {13u, -1, 32u, kQRegs13, kQTypes13, kQNames13},
    {14u, -1, 45u, kQRegs14, kQTypes14, kQNames14},
    {15u, -1, 43u, kQRegs15, kQTypes15, kQNames15},
    {16u, -1, 39u, kQRegs16, kQTypes16, kQNames16},
    {17u, -1, 34u, kQRegs17, kQTypes17, kQNames17},
    {18u, -1, 32u, kQRegs18, kQTypes18, kQNames18},
    {19u, -1, 37u, kQRegs19, kQTypes19, kQNames19},
    {20u, -1, 36u, kQRegs20, kQTypes20, kQNames20},
    {21u, -1, 36u, kQRegs21, kQTypes21, kQNames21},
    {22u, -1, 37u, kQRegs22, kQTypes22, kQNames22},
    {23u, -1, 37u, kQRegs23, kQTypes23, kQNames23},
    {24u, -1, 36u, kQRegs24, kQTypes24, kQNames24},
    {25u, -1, 35u, kQRegs25, kQTypes25, kQNames25},
    {26u, -1, 35u, kQRegs26, kQTypes26, kQNames26},
    {27u, -1, 34u, kQRegs27, kQTypes27, kQNames27},
    {28u, -1, 32u, kQRegs28, kQTypes28, kQNames28},
    {29u, -1, 35u, kQRegs29, kQTypes29, kQNames29},
    {30u, -1, 39u, kQRegs30, kQTypes30, kQNames30},
    {31u, -1, 37u, kQRegs31, kQTypes31, kQNames31},
    {32u, -1, 34u, kQRegs32, kQTypes32, kQNames32},
    {33u, -1, 32u, kQRegs33, kQTypes33, kQNames33},
    {34u, -1, 32u, kQRegs34, kQTypes34, kQNames34},
    {35u, -1, 26u, kQRegs35, kQTypes35, kQNames35},
    {36u, -1, 28u, kQRegs36, kQTypes36, kQNames36},
    {37u, -1, 31u, kQRegs37, kQTypes37, kQNames37},
    {38u, -1, 27u, kQRegs38, kQTypes38, kQNames38},
    {39u, -1, 27u, kQRegs39, kQTypes39, kQNames39},
    {40u, -1, 30u, kQRegs40, kQTypes40, kQNames40},
    {41u, -1, 29u, kQRegs41, kQTypes41, kQNames41},
    {42u, -1, 30u, kQRegs42, kQTypes42, kQNames42},
    {43u, -1, 6u, kQRegs43, kQTypes43, kQNames43},
};
const QueueSegment kSegments[] = {
    {kQOffs0, kQSubs0, kQWidths0, 64ull, 0u, 4u},
    {kQOffs1, kQSubs1, kQWidths1, 184ull, 12u, 16u},
    {kQOffs2, kQSubs2, kQWidths2, 264ull, 12u, 16u},
    {kQOffs3, kQSubs3, kQWidths3, 392ull, 8u, 16u},
    {kQOffs4, kQSubs4, kQWidths4, 536ull, 4u, 8u},
    {kQOffs5, kQSubs5, kQWidths5, 736ull, 4u, 8u},
    {kQOffs6, kQSubs6, kQWidths6, 920ull, 12u, 16u},
    {kQOffs7, kQSubs7, kQWidths7, 1112ull, 12u, 16u},
    {kQOffs8, kQSubs8, kQWidths8, 1304ull, 4u, 8u},
    {kQOffs9, kQSubs9, kQWidths9, 1520ull, 0u, 4u},
    {kQOffs10, kQSubs10, kQWidths10, 1720ull, 4u, 8u},
    {kQOffs11, kQSubs11, kQWidths11, 1888ull, 8u, 16u},
    {kQOffs12, kQSubs12, kQWidths12, 2032ull, 8u, 16u},
    {kQOffs13, kQSubs13, kQWidths13, 2176ull, 0u, 4u},
    {kQOffs14, kQSubs14, kQWidths14, 2360ull, 4u, 8u},
    {kQOffs15, kQSubs15, kQWidths15, 2528ull, 12u, 16u},
    {kQOffs16, kQSubs16, kQWidths16, 2688ull, 12u, 16u},
    {kQOffs17, kQSubs17, kQWidths17, 2832ull, 8u, 16u},
    {kQOffs18, kQSubs18, kQWidths18, 2976ull, 0u, 4u},
    {kQOffs19, kQSubs19, kQWidths19, 3128ull, 4u, 8u},
    {kQOffs20, kQSubs20, kQWidths20, 3280ull, 0u, 4u},
    {kQOffs21, kQSubs21, kQWidths21, 3432ull, 0u, 4u},
    {kQOffs22, kQSubs22, kQWidths22, 3584ull, 4u, 8u},
    {kQOffs23, kQSubs23, kQWidths23, 3736ull, 4u, 8u},
    {kQOffs24, kQSubs24, kQWidths24, 3888ull, 0u, 4u},
    {kQOffs25, kQSubs25, kQWidths25, 4024ull, 12u, 16u},
    {kQOffs26, kQSubs26, kQWidths26, 4168ull, 12u, 16u},
    {kQOffs27, kQSubs27, kQWidths27, 4312ull, 8u, 16u},
    {kQOffs28, kQSubs28, kQWidths28, 4456ull, 0u, 4u},
    {kQOffs29, kQSubs29, kQWidths29, 4592ull, 12u, 16u},
    {kQOffs30, kQSubs30, kQWidths30, 4752ull, 12u, 16u},
    {kQOffs31, kQSubs31, kQWidths31, 4912ull, 4u, 8u},
    {kQOffs32, kQSubs32, kQWidths32, 5048ull, 8u, 16u},
    {kQOffs33, kQSubs33, kQWidths33, 5192ull, 0u, 4u},
    {kQOffs34, kQSubs34, kQWidths34, 5328ull, 0u, 4u},
    {kQOffs35, kQSubs35, kQWidths35, 5432ull, 8u, 16u},
    {kQOffs36, kQSubs36, kQWidths36, 5560ull, 0u, 4u},
    {kQOffs37, kQSubs37, kQWidths37, 5680ull, 12u, 16u},
    {kQOffs38, kQSubs38, kQWidths38, 5792ull, 12u, 16u},
    {kQOffs39, kQSubs39, kQWidths39, 5904ull, 12u, 16u},
    {kQOffs40, kQSubs40, kQWidths40, 6032ull, 8u, 16u},
    {kQOffs41, kQSubs41, kQWidths41, 6160ull, 4u, 8u},
    {kQOffs42, kQSubs42, kQWidths42, 6280ull, 8u, 16u},
    {kQOffs43, kQSubs43, kQWidths43, 6312ull, 8u, 16u},
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

} } // namespace loom_b200::k_pt_const_40

extern const loom_b200::KernelEntry loom_b200_entry_pt_const_40;
const loom_b200::KernelEntry loom_b200_entry_pt_const_40 = {
    &loom_b200::k_pt_const_40::kInfo, loom_b200::k_pt_const_40::K::kRowBytes, 44,
    &loom_b200::k_pt_const_40::launch_plain, &loom_b200::k_pt_const_40::launch_regroup,
    &loom_b200::k_pt_const_40::regroup_occupancy,
    loom_b200::k_pt_const_40::kQueues, loom_b200::k_pt_const_40::kSegments,
    loom_b200::k_pt_const_40::kRegCaps, 8u, loom_b200::k_pt_const_40::K::kMaxStageRow};
