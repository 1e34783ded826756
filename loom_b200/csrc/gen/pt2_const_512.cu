// Generated by loom_b200.codegen from loom_b200/ir/pt2_const_512.lir.
// Kernel IR digest 89a954cc5f4ea54a; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_pt2_const_512 {

__constant__ unsigned kInstrTab[55] = {29, 297, 2, 37, 10, 31, 11, 20, 3, 19, 10, 13, 22, 7, 28, 12, 15, 7, 7, 25, 3, 3, 3, 5, 11, 4, 3, 2, 4, 13, 15, 14, 16, 13, 5, 14, 31, 4, 19, 12, 12, 8, 4, 42, 36, 113, 42, 69, 37, 82, 27, 53, 128, 23, 5};
__constant__ unsigned kLiveTab[55] = {108, 164, 180, 108, 164, 176, 240, 232, 232, 224, 252, 240, 212, 180, 172, 224, 216, 200, 180, 172, 192, 188, 188, 192, 192, 188, 184, 184, 180, 172, 184, 200, 192, 180, 172, 168, 128, 148, 148, 148, 148, 160, 164, 156, 164, 168, 168, 144, 164, 152, 168, 180, 176, 160, 24};
__constant__ int kQueueBlock[55] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54};
__constant__ unsigned kQuorumTab[55] = {1, 25, 0, 5, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 15, 0, 10, 0, 12, 0, 3, 16, 0, 0};
__constant__ unsigned kRankTab[55] = {0, 1, 2, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 34, 35, 30, 31, 32, 33, 36, 37, 38, 39, 40, 41, 42, 43, 46, 49, 53, 52, 51, 50, 54, 11, 7, 44, 45, 10, 6, 9, 8, 3, 4, 5, 47, 48};

struct K
{
    static constexpr int kNumBlocks = 55;
    static constexpr int kNumQueues = 55;
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
        unsigned int r8; // tmp1: f32,u32
        unsigned int r9; // tmp2: f32,u32
        unsigned int r10; // c0: u32
        unsigned int r11; // c1: u32
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
        float r25; // TP0: f32
        float r26; // TP1: f32
        float r27; // TP2: f32
        float r28; // SL0: f32
        float r29; // SL1: f32
        float r30; // SL2: f32
        float r31; // clr0: f32
        float r32; // clr1: f32
        float r33; // clr2: f32
        unsigned int r34; // depth: u32
        float r35; // d2: f32
        float r36; // vr00: f32
        float r37; // vr01: f32
        float r38; // vr02: f32
        float r39; // t: f32
        unsigned int r40; // pid: u32
        unsigned int r41; // rp: u32
        float r42; // vr10: f32
        unsigned int r43; // vr11: u32,f32
        unsigned int r44; // vr12: u32,f32
        float r45; // vr20: f32
        float r46; // vr21: f32
        float r47; // vr22: f32
        unsigned int r48; // vr30: u32,f32
        unsigned int r49; // vr31: u32,f32
        float r50; // vr32: f32
        float r51; // vr40: f32
        float r52; // vr41: f32
        unsigned int r53; // vr42: u32,f32
        float r54; // vr50: f32
        float r55; // vr51: f32
        float r56; // vr52: f32
        unsigned int r57; // hit: u32,f32
        float r58; // vr60: f32
        float r59; // vr61: f32
        float r60; // vr62: f32
        unsigned int r61; // ct: u32,f32
        float r62; // t0: f32
        float r63; // t1: f32
        float r64; // t2: f32
        float r65; // n0: f32
        float r66; // n1: f32
        float r67; // n2: f32
        unsigned int r68; // metal: u32
        float r69; // wi0: f32
        float r70; // wi1: f32
        float r71; // wi2: f32
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
        R.r14 = 0;
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
        R.r33 = 0;
        R.r34 = 0;
        R.r35 = 0;
        R.r61 = 0;
        R.r62 = 0;
        R.r63 = 0;
        R.r64 = 0;
        R.r65 = 0;
        R.r66 = 0;
        R.r67 = 0;
        R.r68 = 0;
        R.r69 = 0;
        R.r70 = 0;
        R.r71 = 0;
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
    static constexpr int kNumLong = 3;
    // j-th long block (most instructions first)
    __device__ __forceinline__ static int long_block(const int j)
    {
        switch(j)
        {
        case 0: return 1;
        case 1: return 52;
        case 2: return 45;
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
        case 44: goto L_B44;
        case 45: goto L_B45;
        case 46: goto L_B46;
        case 47: goto L_B47;
        case 48: goto L_B48;
        case 49: goto L_B49;
        case 50: goto L_B50;
        case 51: goto L_B51;
        case 52: goto L_B52;
        case 53: goto L_B53;
        case 54: goto L_B54;
        default: return kHalt;
        }
    L_B0: // START
        if(stop_heavy && !fresh) return 0;
    L_B0_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 0, 29u);
        R.r6 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r1) >> static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r7 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r1) & static_cast<unsigned int>(((unsigned int)0xffffull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) >> static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r9 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) & static_cast<unsigned int>(((unsigned int)0xffffull))));
        R.r10 = static_cast<unsigned int>(R.r6);
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) * static_cast<unsigned int>(((unsigned int)0x200ull))));
        R.r10 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) + static_cast<unsigned int>(R.r7)));
        R.r11 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r8 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p+9f)));
        R.r9 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p+9f)));
        R.r12 = static_cast<float>(R.r6);
        R.r13 = static_cast<float>(R.r7);
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) / static_cast<float>(bitcast<float>(R.r9)))));
        R.r15 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) / static_cast<float>(bitcast<float>(R.r8))));
        R.r15 = static_cast<float>(static_cast<float>(static_cast<float>(R.r15) * static_cast<float>((0x1.0000000000000p+0f))));
        R.r16 = static_cast<float>((0x0.0p+0f));
        R.r17 = static_cast<float>((0x0.0p+0f));
        R.r12 = static_cast<float>(static_cast<float>(static_cast<float>(R.r12) / static_cast<float>(bitcast<float>(R.r8))));
        R.r12 = static_cast<float>(static_cast<float>(static_cast<float>(R.r12) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r12 = static_cast<float>(static_cast<float>(static_cast<float>(R.r12) * static_cast<float>(bitcast<float>(R.r14))));
        R.r13 = static_cast<float>(static_cast<float>(static_cast<float>(R.r13) / static_cast<float>(bitcast<float>(R.r9))));
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
        if constexpr(kProf) count_block(ctx, 1, 297u);
        R.r20 = static_cast<unsigned int>(R.r10);
        R.r21 = static_cast<unsigned int>(R.r11);
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x3ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0xba0beefull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x7ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(R.r21)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) << static_cast<unsigned int>(R.r14)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(R.r8)));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) | static_cast<unsigned int>(R.r8)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) ^ static_cast<unsigned int>(R.r20)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) + static_cast<unsigned int>(((unsigned int)0x4a06042ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0xf00deadull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) + static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r10) + static_cast<unsigned int>(((unsigned int)0x2611501ull))));
        R.r8 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r14) < static_cast<unsigned int>(R.r10)));
        R.r9 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r11) + static_cast<unsigned int>(R.r14)));
        R.r11 = static_cast<unsigned int>(((R.r8) ? (R.r9) : (R.r11)));
        R.r10 = static_cast<unsigned int>(((R.r8) ? (((unsigned int)0x0ull)) : (R.r14)));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) >> static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) | static_cast<unsigned int>(((unsigned int)0x3f800000ull))));
        R.r20 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) - static_cast<float>((0x1.0000000000000p+0f)))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) >> static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r21) | static_cast<unsigned int>(((unsigned int)0x3f800000ull))));
        R.r21 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r21)) - static_cast<float>((0x1.0000000000000p+0f)))));
        R.r14 = static_cast<unsigned int>(op_min<unsigned int>(static_cast<unsigned int>(R.r18), static_cast<unsigned int>(((unsigned int)0x4ull))));
        switch(R.r14) {
        case 0: goto L_B3;
        case 1: goto L_B42;
        case 2: goto L_B46;
        case 3: goto L_B48;
        case 4: goto L_B2;
        default: goto L_HALT;
        }
    L_B2: // roll_split
        fresh = false;
        if constexpr(kProf) count_block(ctx, 2, 2u);
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) - static_cast<unsigned int>(((unsigned int)0x4ull))));
        switch(R.r18) {
        case 0: goto L_B49;
        case 1: goto L_B43;
        case 2: goto L_B47;
        case 3: goto L_B45;
        case 4: goto L_B50;
        default: goto L_HALT;
        }
    L_B3: // sample_pixel
        if(stop_heavy && !fresh) return 3;
    L_B3_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 3, 37u);
        R.r22 = static_cast<float>((0x0.0p+0f));
        R.r23 = static_cast<float>((0x0.0p+0f));
        R.r24 = static_cast<float>((0x1.0000000000000p+1f));
        R.r25 = static_cast<float>((0x1.0000000000000p+0f));
        R.r26 = static_cast<float>((0x1.0000000000000p+0f));
        R.r27 = static_cast<float>((0x1.0000000000000p+0f));
        R.r28 = static_cast<float>((0x0.0p+0f));
        R.r29 = static_cast<float>((0x0.0p+0f));
        R.r30 = static_cast<float>((0x0.0p+0f));
        R.r6 = bitcast<unsigned int>(static_cast<float>(R.r12));
        R.r7 = bitcast<unsigned int>(static_cast<float>(R.r13));
        R.r31 = static_cast<float>((0x0.0p+0f));
        R.r32 = static_cast<float>((0x0.0p+0f));
        R.r33 = static_cast<float>((0x0.0p+0f));
        R.r34 = static_cast<unsigned int>(((unsigned int)0x0ull));
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
        R.r35 = static_cast<float>((-0x1.0000000000000p+0f));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r35, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r14))));
        goto L_B4;
    L_B4: // traverse_scene
        fresh = false;
        if constexpr(kProf) count_block(ctx, 4, 10u);
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>((0x1.0624de0000000p-10f))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>((0x1.0624de0000000p-10f))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>((0x1.0624de0000000p-10f))));
        R.r22 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) + static_cast<float>(R.r36)));
        R.r23 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) + static_cast<float>(R.r37)));
        R.r24 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) + static_cast<float>(R.r38)));
        R.r39 = static_cast<float>((0x1.e848000000000p+19f));
        R.r40 = static_cast<unsigned int>(((unsigned int)0xcull));
        R.r41 = static_cast<unsigned int>(((unsigned int)0x0ull));
        goto L_B5;
    L_B5: // traverse_box
        if(budget == 0u) return 5;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 5, 31u);
        R.r36 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : ((R.r41) == 2 ? (0x1.0000000000000p+0f) : ((R.r41) == 3 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r37 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : ((R.r41) == 2 ? (-0x1.0000000000000p+0f) : ((R.r41) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r38 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (0x1.0000000000000p+0f) : ((R.r41) == 1 ? (0x1.0000000000000p+0f) : ((R.r41) == 2 ? (-0x1.0000000000000p+0f) : ((R.r41) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r42 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : ((R.r41) == 2 ? (0x1.0000000000000p+0f) : ((R.r41) == 3 ? (-0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : ((R.r41) == 2 ? (-0x1.0000000000000p+0f) : ((R.r41) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f))))))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r41) == 0 ? (0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : ((R.r41) == 2 ? (0x1.0000000000000p+0f) : ((R.r41) == 3 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f))))))));
        R.r45 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : ((R.r41) == 2 ? (0x1.0000000000000p+0f) : ((R.r41) == 3 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r46 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (0x1.0000000000000p+0f) : ((R.r41) == 2 ? (0x1.0000000000000p+0f) : ((R.r41) == 3 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f)))))));
        R.r47 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : ((R.r41) == 2 ? (0x1.0000000000000p+0f) : ((R.r41) == 3 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : ((R.r41) == 2 ? (0x1.0000000000000p+0f) : ((R.r41) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f))))))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (0x1.0000000000000p+0f) : ((R.r41) == 2 ? (0x1.0000000000000p+0f) : ((R.r41) == 3 ? (0x1.0000000000000p+0f) : (0x1.0000000000000p+0f))))))));
        R.r50 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (0x1.0000000000000p+0f) : ((R.r41) == 2 ? (-0x1.0000000000000p+0f) : ((R.r41) == 3 ? (0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) - static_cast<float>(R.r36)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) - static_cast<float>(R.r37)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r50) - static_cast<float>(R.r38))));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r36)));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) - static_cast<float>(R.r37)));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r44)) - static_cast<float>(R.r38)));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(R.r55))));
        R.r58 = static_cast<float>(op_fma(bitcast<float>(R.r7), R.r56, (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r56))));
        R.r59 = static_cast<float>(op_fma(R.r35, R.r54, (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r54))));
        R.r60 = static_cast<float>(op_fma(bitcast<float>(R.r6), R.r55, (-(bitcast<float>(R.r57)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r51, R.r58, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r52, R.r59, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r53), R.r60, bitcast<float>(R.r14))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r14)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r8)) >= static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r57) goto L_B6; else goto L_B13;
    L_B6: // isect_quad_l1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 6, 11u);
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r36)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r37)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r38))));
        R.r8 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r51, R.r58, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r52, R.r59, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r53), R.r60, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r8)) >= static_cast<float>((0x0.0p+0f))));
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r8)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r57) goto L_B7; else goto L_B13;
    L_B7: // isect_quad_l2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 7, 20u);
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) - static_cast<float>(R.r36)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) - static_cast<float>(R.r37)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r50) - static_cast<float>(R.r38))));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r36)));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r37)));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r38)));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r56) * static_cast<float>(R.r52))));
        R.r58 = static_cast<float>(op_fma(R.r55, bitcast<float>(R.r53), (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r54) * static_cast<float>(bitcast<float>(R.r53)))));
        R.r59 = static_cast<float>(op_fma(R.r56, R.r51, (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r55) * static_cast<float>(R.r51))));
        R.r60 = static_cast<float>(op_fma(R.r54, R.r52, (-(bitcast<float>(R.r57)))));
        R.r9 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r58, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r59, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r60, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r9)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r9)) >= static_cast<float>((0x0.0p+0f))));
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r9)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r57) goto L_B8; else goto L_B13;
    L_B8: // isect_quad_l3
        fresh = false;
        if constexpr(kProf) count_block(ctx, 8, 3u);
        R.r61 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) + static_cast<float>(bitcast<float>(R.r9)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r61)) > static_cast<float>((0x1.0000000000000p+0f))));
        if(R.r57) goto L_B9; else goto L_B12;
    L_B9: // isect_quad_l4
        fresh = false;
        if constexpr(kProf) count_block(ctx, 9, 19u);
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r45)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) - static_cast<float>(R.r46)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r44)) - static_cast<float>(R.r47))));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) - static_cast<float>(R.r45)));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) - static_cast<float>(R.r46)));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) - static_cast<float>(R.r47)));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(R.r55))));
        R.r58 = static_cast<float>(op_fma(bitcast<float>(R.r7), R.r56, (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r56))));
        R.r59 = static_cast<float>(op_fma(R.r35, R.r54, (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r54))));
        R.r60 = static_cast<float>(op_fma(bitcast<float>(R.r6), R.r55, (-(bitcast<float>(R.r57)))));
        R.r61 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r51, R.r58, bitcast<float>(R.r61))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r52, R.r59, bitcast<float>(R.r61))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r53), R.r60, bitcast<float>(R.r61))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r61)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r57)) >= static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r57) goto L_B10; else goto L_B13;
    L_B10: // isect_quad_l5
        fresh = false;
        if constexpr(kProf) count_block(ctx, 10, 10u);
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r45)));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r46)));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r47)));
        R.r57 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r54, R.r58, bitcast<float>(R.r57))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r55, R.r59, bitcast<float>(R.r57))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r56, R.r60, bitcast<float>(R.r57))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r57)) / static_cast<float>(bitcast<float>(R.r61)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r57)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r57) goto L_B11; else goto L_B13;
    L_B11: // isect_quad_l6
        fresh = false;
        if constexpr(kProf) count_block(ctx, 11, 13u);
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r56) * static_cast<float>(R.r52))));
        R.r58 = static_cast<float>(op_fma(R.r55, bitcast<float>(R.r53), (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r54) * static_cast<float>(bitcast<float>(R.r53)))));
        R.r59 = static_cast<float>(op_fma(R.r56, R.r51, (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r55) * static_cast<float>(R.r51))));
        R.r60 = static_cast<float>(op_fma(R.r54, R.r52, (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r58, bitcast<float>(R.r57))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r59, bitcast<float>(R.r57))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r60, bitcast<float>(R.r57))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r57)) / static_cast<float>(bitcast<float>(R.r61)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r57)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r57) goto L_B12; else goto L_B13;
    L_B12: // isect_quad_l7
        fresh = false;
        if constexpr(kProf) count_block(ctx, 12, 22u);
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) - static_cast<float>(R.r36))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) - static_cast<float>(R.r37))));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) - static_cast<float>(R.r38)));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r36)));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r37)));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r38)));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r56) * static_cast<float>(bitcast<float>(R.r49)))));
        R.r58 = static_cast<float>(op_fma(R.r55, R.r50, (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r54) * static_cast<float>(R.r50))));
        R.r59 = static_cast<float>(op_fma(R.r56, bitcast<float>(R.r48), (-(bitcast<float>(R.r57)))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r55) * static_cast<float>(bitcast<float>(R.r48)))));
        R.r60 = static_cast<float>(op_fma(R.r54, bitcast<float>(R.r49), (-(bitcast<float>(R.r57)))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r36)));
        R.r43 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) - static_cast<float>(R.r37))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r44)) - static_cast<float>(R.r38))));
        R.r61 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r42, R.r58, bitcast<float>(R.r61))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r43), R.r59, bitcast<float>(R.r61))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r44), R.r60, bitcast<float>(R.r61))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r61)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r61)) >= static_cast<float>((0x0.0p+0f))));
        goto L_B13;
    L_B13: // isect_quad_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 13, 7u);
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r61)) < static_cast<float>(R.r39))));
        R.r39 = static_cast<float>(((R.r57) ? (bitcast<float>(R.r61)) : (R.r39)));
        R.r40 = static_cast<unsigned int>(((R.r57) ? (R.r41) : (R.r40)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r41) == static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r41 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r41) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r41 = static_cast<unsigned int>(((R.r14) ? (((unsigned int)0x0ull)) : (R.r41)));
        if(R.r14) goto L_B14; else goto L_B5;
    L_B14: // traverse_tetrahedron
        if(budget == 0u) return 14;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 14, 28u);
        R.r36 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.935f360000000p-1f) : ((R.r41) == 1 ? (-0x1.157b7e0000000p-1f) : (0x1.09d1420000000p-3f)))));
        R.r37 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f)))));
        R.r38 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.2cf8d20000000p-1f) : ((R.r41) == 1 ? (0x1.51b56e0000000p-2f) : (-0x1.5e2a2e0000000p-2f)))));
        R.r42 = static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.157b7e0000000p-1f) : ((R.r41) == 1 ? (0x1.09d1420000000p-3f) : (-0x1.935f360000000p-1f)))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r41) == 0 ? (-0x1.0000000000000p+0f) : ((R.r41) == 1 ? (-0x1.0000000000000p+0f) : (-0x1.0000000000000p+0f))))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(((R.r41) == 0 ? (0x1.51b56e0000000p-2f) : ((R.r41) == 1 ? (-0x1.5e2a2e0000000p-2f) : (-0x1.2cf8d20000000p-1f))))));
        R.r45 = static_cast<float>((-0x1.9999980000000p-2f));
        R.r46 = static_cast<float>((-0x1.6b0f960000000p-3f));
        R.r47 = static_cast<float>((-0x1.9999980000000p-3f));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) - static_cast<float>(R.r36)));
        R.r43 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) - static_cast<float>(R.r37))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r44)) - static_cast<float>(R.r38))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) - static_cast<float>(R.r36)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>(R.r37)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) - static_cast<float>(R.r38)));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(R.r46))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r47, (-(bitcast<float>(R.r57))))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r47))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r45, (-(bitcast<float>(R.r57))))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r45))));
        R.r50 = static_cast<float>(op_fma(bitcast<float>(R.r6), R.r46, (-(bitcast<float>(R.r57)))));
        R.r61 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r42, bitcast<float>(R.r48), bitcast<float>(R.r61))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r43), bitcast<float>(R.r49), bitcast<float>(R.r61))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r44), R.r50, bitcast<float>(R.r61))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r61)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r57) goto L_B15; else goto L_B18;
    L_B15: // isect_triangle_mid1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 15, 12u);
        R.r61 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(bitcast<float>(R.r61)))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r36)));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r37)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r38)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r36, bitcast<float>(R.r48), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r37, bitcast<float>(R.r49), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, R.r50, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r61)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x0.0p+0f))));
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r57) goto L_B16; else goto L_B18;
    L_B16: // isect_triangle_mid2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 16, 15u);
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>(bitcast<float>(R.r43)))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r37, bitcast<float>(R.r44), (-(bitcast<float>(R.r8))))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(bitcast<float>(R.r44)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, R.r42, (-(bitcast<float>(R.r8))))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r37) * static_cast<float>(R.r42))));
        R.r50 = static_cast<float>(op_fma(R.r36, bitcast<float>(R.r43), (-(bitcast<float>(R.r8)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r48), bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r49), bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r50, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) * static_cast<float>(bitcast<float>(R.r61)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r8)) >= static_cast<float>((0x0.0p+0f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) + static_cast<float>(bitcast<float>(R.r8)))));
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) <= static_cast<float>((0x1.0000000000000p+0f)))));
        if(R.r57) goto L_B17; else goto L_B18;
    L_B17: // isect_triangle_mid3
        fresh = false;
        if constexpr(kProf) count_block(ctx, 17, 7u);
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, bitcast<float>(R.r48), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, bitcast<float>(R.r49), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, R.r50, bitcast<float>(R.r14))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r61)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r61)) > static_cast<float>((0x0.0p+0f))));
        goto L_B18;
    L_B18: // isect_triangle_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 18, 7u);
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r61)) < static_cast<float>(R.r39))));
        R.r39 = static_cast<float>(((R.r57) ? (bitcast<float>(R.r61)) : (R.r39)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r41) + static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r40 = static_cast<unsigned int>(((R.r57) ? (R.r8) : (R.r40)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r41) == static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r41 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r41) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        if(R.r14) goto L_B19; else goto L_B14;
    L_B19: // traverse_sphere
        fresh = false;
        if constexpr(kProf) count_block(ctx, 19, 25u);
        R.r36 = static_cast<float>((0x1.99999a0000000p-4f));
        R.r37 = static_cast<float>((-0x1.6666660000000p-1f));
        R.r38 = static_cast<float>((0x1.3333340000000p-2f));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>(R.r36)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>(R.r37)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>(R.r38)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.3333340000000p-2f)) * static_cast<float>((0x1.3333340000000p-2f)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r45, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, R.r46, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, R.r47, bitcast<float>(R.r8))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) - static_cast<float>(bitcast<float>(R.r14)))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r43 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r43 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r45, bitcast<float>(R.r43))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r46, bitcast<float>(R.r43))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r47, bitcast<float>(R.r43))));
        R.r42 = static_cast<float>((0x0.0p+0f));
        R.r42 = static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), R.r42));
        R.r42 = static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), R.r42));
        R.r42 = static_cast<float>(op_fma(R.r35, R.r35, R.r42));
        R.r41 = static_cast<unsigned int>(((unsigned int)0x8ull));
        goto L_B20;
    L_B20: // traverse_solve_quadratic
        if(budget == 0u) return 20;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 20, 3u);
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(R.r42))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r57)) > static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r57) goto L_B23; else goto L_B21;
    L_B21: // sq_head1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 21, 3u);
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r43)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r57)) > static_cast<float>((0x1.a36e2e0000000p-14f))));
        if(R.r57) goto L_B22; else goto L_B27;
    L_B22: // sq_head2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 22, 3u);
        R.r61 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r44)))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r61)) / static_cast<float>(bitcast<float>(R.r43)))));
        goto L_B27;
    L_B23: // sq_mid1
        fresh = false;
        if constexpr(kProf) count_block(ctx, 23, 5u);
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r44)) * static_cast<float>(R.r42))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>((0x1.0000000000000p+2f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r43), bitcast<float>(R.r43), (-(bitcast<float>(R.r14))))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r57) goto L_B24; else goto L_B27;
    L_B24: // sq_mid2
        fresh = false;
        if constexpr(kProf) count_block(ctx, 24, 11u);
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r61 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r43)) < static_cast<float>((0x0.0p+0f))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) - static_cast<float>(bitcast<float>(R.r57)))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) + static_cast<float>(bitcast<float>(R.r57)))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(((R.r61) ? (bitcast<float>(R.r8)) : (bitcast<float>(R.r43)))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) * static_cast<float>((-0x1.0000000000000p-1f)))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) / static_cast<float>(R.r42))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r44)) / static_cast<float>(bitcast<float>(R.r43)))));
        R.r43 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r61)) < static_cast<float>((0x0.0p+0f))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(((R.r43) ? (bitcast<float>(R.r44)) : (bitcast<float>(R.r61)))));
        if(R.r43) goto L_B26; else goto L_B25;
    L_B25: // sq_mid
        fresh = false;
        if constexpr(kProf) count_block(ctx, 25, 4u);
        R.r43 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r44)) < static_cast<float>((0x0.0p+0f))));
        R.r57 = bitcast<unsigned int>(static_cast<float>(op_min<float>(static_cast<float>(bitcast<float>(R.r61)), static_cast<float>(bitcast<float>(R.r44)))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(((R.r43) ? (bitcast<float>(R.r61)) : (bitcast<float>(R.r57)))));
        goto L_B26;
    L_B26: // sq_tail
        fresh = false;
        if constexpr(kProf) count_block(ctx, 26, 3u);
        R.r57 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r61)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r57)) >= static_cast<float>((0x0.0p+0f))));
        goto L_B27;
    L_B27: // sq_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 27, 2u);
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r41) == static_cast<unsigned int>(((unsigned int)0x8ull))));
        if(R.r14) goto L_B28; else goto L_B30;
    L_B28: // traverse_sphere_fin
        fresh = false;
        if constexpr(kProf) count_block(ctx, 28, 4u);
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r61)) < static_cast<float>(R.r39))));
        R.r39 = static_cast<float>(((R.r57) ? (bitcast<float>(R.r61)) : (R.r39)));
        R.r40 = static_cast<unsigned int>(((R.r57) ? (R.r41) : (R.r40)));
        goto L_B29;
    L_B29: // traverse_cylinder
        fresh = false;
        if constexpr(kProf) count_block(ctx, 29, 13u);
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>((-0x1.0000000000000p+0f))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>((-0x1.3333340000000p-2f))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(R.r35)));
        R.r42 = static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), R.r42));
        R.r43 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>(R.r35))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r36, bitcast<float>(R.r6), bitcast<float>(R.r43))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p-2f)) * static_cast<float>((0x1.0000000000000p-2f)))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, R.r38, (-(bitcast<float>(R.r44))))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r36, R.r36, bitcast<float>(R.r44))));
        R.r41 = static_cast<unsigned int>(((unsigned int)0x9ull));
        goto L_B20;
    L_B30: // traverse_cylinder_fin
        fresh = false;
        if constexpr(kProf) count_block(ctx, 30, 15u);
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r61), R.r37)));
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) >= static_cast<float>((0x0.0p+0f)))));
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r14)) <= static_cast<float>((0x1.4ccccc0000000p-1f)))));
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r61)) < static_cast<float>(R.r39))));
        R.r39 = static_cast<float>(((R.r57) ? (bitcast<float>(R.r61)) : (R.r39)));
        R.r40 = static_cast<unsigned int>(((R.r57) ? (R.r41) : (R.r40)));
        R.r41 = static_cast<unsigned int>(((unsigned int)0xaull));
        R.r36 = static_cast<float>((0x1.0000000000000p-1f));
        R.r37 = static_cast<float>((-0x1.6666660000000p-2f));
        R.r38 = static_cast<float>((-0x1.3333340000000p-2f));
        R.r42 = static_cast<float>((0x0.0p+0f));
        R.r43 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p+0f)));
        R.r44 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x1.0000000000000p-2f)));
        goto L_B31;
    L_B31: // traverse_disk
        if(budget == 0u) return 31;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 31, 14u);
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) - static_cast<float>(R.r22)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) - static_cast<float>(R.r23)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) - static_cast<float>(R.r24)));
        R.r61 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r42, bitcast<float>(R.r61))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, bitcast<float>(R.r43), bitcast<float>(R.r61))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, bitcast<float>(R.r44), bitcast<float>(R.r61))));
        R.r8 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r42, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r43), bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, bitcast<float>(R.r44), bitcast<float>(R.r8))));
        R.r61 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r61)) / static_cast<float>(bitcast<float>(R.r8)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r61)) >= static_cast<float>((0x0.0p+0f))));
        if(R.r57) goto L_B32; else goto L_B33;
    L_B32: // isect_disk_rest
        fresh = false;
        if constexpr(kProf) count_block(ctx, 32, 16u);
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r61))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r61))));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r61))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) + static_cast<float>(R.r22)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) + static_cast<float>(R.r23)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) + static_cast<float>(R.r24)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) - static_cast<float>(R.r36)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>(R.r37)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) - static_cast<float>(R.r38)));
        R.r8 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r45, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, R.r46, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, R.r47, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r8)))));
        R.r57 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r8)) < static_cast<float>(bitcast<float>(R.r14))));
        goto L_B33;
    L_B33: // isect_disk_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 33, 13u);
        R.r57 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r57) && static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r61)) < static_cast<float>(R.r39))));
        R.r39 = static_cast<float>(((R.r57) ? (bitcast<float>(R.r61)) : (R.r39)));
        R.r40 = static_cast<unsigned int>(((R.r57) ? (R.r41) : (R.r40)));
        R.r8 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r41) == static_cast<unsigned int>(((unsigned int)0xbull))));
        R.r41 = static_cast<unsigned int>(((unsigned int)0xbull));
        R.r36 = static_cast<float>((0x0.0p+0f));
        R.r37 = static_cast<float>((0x1.fff2e40000000p-1f));
        R.r38 = static_cast<float>((0x0.0p+0f));
        R.r42 = static_cast<float>((0x0.0p+0f));
        R.r43 = bitcast<unsigned int>(static_cast<float>((-0x1.0000000000000p+0f)));
        R.r44 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x1.6666660000000p-2f)));
        if(R.r8) goto L_B34; else goto L_B31;
    L_B34: // traverse_room_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 34, 5u);
        R.r5 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r5) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r36 = static_cast<float>((0x0.0p+0f));
        R.r37 = static_cast<float>((0x0.0p+0f));
        R.r38 = static_cast<float>((0x0.0p+0f));
        if(R.r18) goto L_B44; else goto L_B35;
    L_B35: // radiance
        fresh = false;
        if constexpr(kProf) count_block(ctx, 35, 14u);
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0xbull))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(((R.r14) ? ((0x1.4000000000000p+2f)) : ((0x0.0p+0f)))));
        R.r9 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0xcull))));
        R.r9 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r9) || static_cast<unsigned int>(static_cast<unsigned int>(R.r34) >= static_cast<unsigned int>(((unsigned int)0x2ull)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(((R.r9) ? ((0x0.0p+0f)) : (bitcast<float>(R.r8)))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r25) * static_cast<float>(bitcast<float>(R.r8))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r26) * static_cast<float>(bitcast<float>(R.r8))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(bitcast<float>(R.r8))));
        R.r28 = static_cast<float>(static_cast<float>(static_cast<float>(R.r28) + static_cast<float>(R.r36)));
        R.r29 = static_cast<float>(static_cast<float>(static_cast<float>(R.r29) + static_cast<float>(R.r37)));
        R.r30 = static_cast<float>(static_cast<float>(static_cast<float>(R.r30) + static_cast<float>(R.r38)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r14) || static_cast<unsigned int>(R.r9)));
        R.r34 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r34) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        if(R.r14) goto L_B53; else goto L_B36;
    L_B36: // set_materials
        fresh = false;
        if constexpr(kProf) count_block(ctx, 36, 31u);
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r39)));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r39)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(R.r39)));
        R.r22 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) + static_cast<float>(R.r36)));
        R.r23 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) + static_cast<float>(R.r37)));
        R.r24 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) + static_cast<float>(R.r38)));
        R.r14 = static_cast<unsigned int>(op_min<unsigned int>(static_cast<unsigned int>(R.r40), static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r31 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.0000000000000p+0f) : ((R.r14) == 1 ? (0x1.0000000000000p+0f) : ((R.r14) == 2 ? (0x1.99999a0000000p-3f) : ((R.r14) == 3 ? (0x1.0000000000000p+0f) : ((R.r14) == 4 ? (0x1.0000000000000p+0f) : (0x0.0p+0f))))))));
        R.r32 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.0000000000000p+0f) : ((R.r14) == 1 ? (0x1.99999a0000000p-2f) : ((R.r14) == 2 ? (0x1.0000000000000p+0f) : ((R.r14) == 3 ? (0x1.0000000000000p+0f) : ((R.r14) == 4 ? (0x1.0000000000000p+0f) : (0x1.b22d100000000p-3f))))))));
        R.r33 = static_cast<float>(static_cast<float>(((R.r14) == 0 ? (0x1.0000000000000p+0f) : ((R.r14) == 1 ? (0x1.99999a0000000p-3f) : ((R.r14) == 2 ? (0x1.99999a0000000p-2f) : ((R.r14) == 3 ? (0x1.0000000000000p+0f) : ((R.r14) == 4 ? (0x1.0000000000000p+0f) : (0x1.1b22d20000000p-1f))))))));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r31 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : (R.r31)));
        R.r32 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : (R.r32)));
        R.r33 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : (R.r33)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) || static_cast<unsigned int>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0xaull)))));
        R.r31 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : (R.r31)));
        R.r32 = static_cast<float>(((R.r14) ? ((0x1.a76c8c0000000p-1f)) : (R.r32)));
        R.r33 = static_cast<float>(((R.r14) ? ((0x1.12f1aa0000000p-1f)) : (R.r33)));
        R.r62 = static_cast<float>((0x0.0p+0f));
        R.r63 = static_cast<float>((0x1.0000000000000p+0f));
        R.r64 = static_cast<float>((0x0.0p+0f));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0xaull))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) || static_cast<unsigned int>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0xbull)))));
        R.r8 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) || static_cast<unsigned int>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0x9ull)))));
        R.r41 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r41 = static_cast<unsigned int>(((R.r14) ? (((unsigned int)0x1ull)) : (R.r41)));
        R.r9 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r40) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r41 = static_cast<unsigned int>(((R.r8) ? (R.r9) : (R.r41)));
        switch(R.r41) {
        case 0: goto L_B37;
        case 1: goto L_B38;
        case 2: goto L_B39;
        case 3: goto L_B40;
        default: goto L_HALT;
        }
    L_B37: // set_polygon_normal
        fresh = false;
        if constexpr(kProf) count_block(ctx, 37, 4u);
        R.r65 = static_cast<float>(static_cast<float>(((R.r40) == 0 ? (0x0.0p+0f) : ((R.r40) == 1 ? (0x1.0000000000000p+0f) : ((R.r40) == 2 ? (-0x1.0000000000000p+0f) : ((R.r40) == 3 ? (0x0.0p+0f) : ((R.r40) == 4 ? (0x0.0p+0f) : ((R.r40) == 5 ? (-0x1.d52cd80000000p-1f) : ((R.r40) == 6 ? (0x1.5775c60000000p-1f) : (0x1.f6dc440000000p-3f))))))))));
        R.r66 = static_cast<float>(static_cast<float>(((R.r40) == 0 ? (0x1.0000000000000p+0f) : ((R.r40) == 1 ? (0x0.0p+0f) : ((R.r40) == 2 ? (0x0.0p+0f) : ((R.r40) == 3 ? (-0x1.0000000000000p+0f) : ((R.r40) == 4 ? (0x0.0p+0f) : ((R.r40) == 5 ? (0x1.43d1320000000p-2f) : ((R.r40) == 6 ? (0x1.43d1360000000p-2f) : (0x1.43d1360000000p-2f))))))))));
        R.r67 = static_cast<float>(static_cast<float>(((R.r40) == 0 ? (0x0.0p+0f) : ((R.r40) == 1 ? (0x0.0p+0f) : ((R.r40) == 2 ? (0x0.0p+0f) : ((R.r40) == 3 ? (0x0.0p+0f) : ((R.r40) == 4 ? (0x1.0000000000000p+0f) : ((R.r40) == 5 ? (0x1.f6dc380000000p-3f) : ((R.r40) == 6 ? (0x1.5775c60000000p-1f) : (-0x1.d52cd40000000p-1f))))))))));
        goto L_B41;
    L_B38: // set_disk_normal
        fresh = false;
        if constexpr(kProf) count_block(ctx, 38, 19u);
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0xaull))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>((-0x1.6666660000000p-2f))));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>((-0x1.3333340000000p-2f))));
        R.r8 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r45, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, R.r46, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, R.r47, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r8)))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) * static_cast<float>(bitcast<float>(R.r8))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>(bitcast<float>(R.r8))));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) * static_cast<float>(bitcast<float>(R.r8))));
        R.r65 = static_cast<float>((0x0.0p+0f));
        R.r66 = static_cast<float>(((R.r14) ? ((0x1.0000000000000p+0f)) : ((-0x1.0000000000000p+0f))));
        R.r67 = static_cast<float>((0x0.0p+0f));
        R.r62 = static_cast<float>(((R.r14) ? (R.r45) : (R.r62)));
        R.r63 = static_cast<float>(((R.r14) ? (R.r46) : (R.r63)));
        R.r64 = static_cast<float>(((R.r14) ? (R.r47) : (R.r64)));
        goto L_B41;
    L_B39: // compute_sphere_normal
        fresh = false;
        if constexpr(kProf) count_block(ctx, 39, 12u);
        R.r65 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>((0x1.99999a0000000p-4f))));
        R.r66 = static_cast<float>(static_cast<float>(static_cast<float>(R.r23) - static_cast<float>((-0x1.6666660000000p-1f))));
        R.r67 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>((0x1.3333340000000p-2f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r65, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r66, R.r66, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r67, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r65 = static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(bitcast<float>(R.r14))));
        R.r66 = static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>(bitcast<float>(R.r14))));
        R.r67 = static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>(bitcast<float>(R.r14))));
        goto L_B41;
    L_B40: // compute_cylinder_normal
        fresh = false;
        if constexpr(kProf) count_block(ctx, 40, 12u);
        R.r66 = static_cast<float>((0x0.0p+0f));
        R.r65 = static_cast<float>(static_cast<float>(static_cast<float>(R.r22) - static_cast<float>((0x1.0000000000000p-1f))));
        R.r67 = static_cast<float>(static_cast<float>(static_cast<float>(R.r24) - static_cast<float>((-0x1.3333340000000p-2f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r65, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r66, R.r66, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r67, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r65 = static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(bitcast<float>(R.r14))));
        R.r66 = static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>(bitcast<float>(R.r14))));
        R.r67 = static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>(bitcast<float>(R.r14))));
        goto L_B41;
    L_B41: // set_materials_end
        fresh = false;
        if constexpr(kProf) count_block(ctx, 41, 8u);
        R.r18 = static_cast<unsigned int>(((unsigned int)0x1ull));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) < static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r40) - static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r8 = static_cast<unsigned int>(op_min<unsigned int>(static_cast<unsigned int>(R.r8), static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r9 = static_cast<unsigned int>(static_cast<unsigned int>(((R.r8) == 0 ? ((unsigned int)0x2ull) : ((R.r8) == 1 ? ((unsigned int)0x3ull) : ((R.r8) == 2 ? ((unsigned int)0x3ull) : ((R.r8) == 3 ? ((unsigned int)0x3ull) : ((R.r8) == 4 ? ((unsigned int)0x4ull) : ((R.r8) == 5 ? ((unsigned int)0x1ull) : ((unsigned int)0x1ull)))))))));
        R.r68 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) > static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r18 = static_cast<unsigned int>(((R.r14) ? (R.r18) : (R.r9)));
        goto L_B1;
    L_B42: // test_direct
        fresh = false;
        if constexpr(kProf) count_block(ctx, 42, 4u);
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r20)) < static_cast<float>((0x1.0000000000000p-1f))));
        R.r8 = static_cast<unsigned int>(((R.r68) ? (((unsigned int)0x8ull)) : (((unsigned int)0x6ull))));
        R.r18 = static_cast<unsigned int>(((R.r14) ? (((unsigned int)0x5ull)) : (R.r8)));
        goto L_B1;
    L_B43: // direct
        if(stop_heavy && !fresh) return 43;
    L_B43_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 43, 42u);
        R.r69 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r6))));
        R.r70 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r7))));
        R.r71 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r35)));
        R.r20 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r20)))));
        R.r20 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) * static_cast<float>((0x1.6666660000000p-2f)))));
        R.r21 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r21)) - static_cast<float>((0x1.0000000000000p-1f)))));
        R.r21 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r21)) * static_cast<float>((0x1.921fb60000000p+2f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_sin(static_cast<float>(bitcast<float>(R.r21)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r20)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x0.0p+0f)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>((0x0.0p+0f)) * static_cast<float>(bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_cos(static_cast<float>(bitcast<float>(R.r21)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r20)))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>((0x0.0p+0f)) * static_cast<float>(bitcast<float>(R.r14))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>((0x0.0p+0f)) * static_cast<float>(bitcast<float>(R.r14))));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) * static_cast<float>(bitcast<float>(R.r14))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) + static_cast<float>(R.r45))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) + static_cast<float>(R.r46))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) + static_cast<float>(R.r47)));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) + static_cast<float>((0x0.0p+0f)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) + static_cast<float>((0x1.fff2e40000000p-1f)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) + static_cast<float>((0x0.0p+0f))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) - static_cast<float>(R.r22))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) - static_cast<float>(R.r23))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) - static_cast<float>(R.r24)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r35, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r65, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r66, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r67, bitcast<float>(R.r14))));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) > static_cast<float>((0x0.0p+0f))));
        R.r8 = static_cast<unsigned int>(((R.r68) ? (((unsigned int)0x8ull)) : (((unsigned int)0x6ull))));
        R.r18 = static_cast<unsigned int>(((R.r14) ? (((unsigned int)0x1ull)) : (R.r8)));
        if(R.r14) goto L_B4; else goto L_B1;
    L_B44: // direct_pdf
        fresh = false;
        if constexpr(kProf) count_block(ctx, 44, 36u);
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>((0x0.0p+0f)) - static_cast<float>(R.r22)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.fff2e40000000p-1f)) - static_cast<float>(R.r23)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>((0x0.0p+0f)) - static_cast<float>(R.r24)));
        R.r8 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r45, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, R.r46, bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, R.r47, bitcast<float>(R.r8))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma((0x0.0p+0f), bitcast<float>(R.r6), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma((-0x1.0000000000000p+0f), bitcast<float>(R.r7), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma((0x0.0p+0f), R.r35, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r14)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>((0x1.8a14d40000000p-2f)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) / static_cast<float>(bitcast<float>(R.r14)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r65, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r66, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r67, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_max<float>(static_cast<float>(bitcast<float>(R.r14)), static_cast<float>((0x0.0p+0f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>((0x1.4000000000000p+2f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) / static_cast<float>(bitcast<float>(R.r8)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) / static_cast<float>((0x1.0000000000000p-1f)))));
        R.r9 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r40) == static_cast<unsigned int>(((unsigned int)0xbull))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(((R.r68) ? ((0x0.0p+0f)) : (bitcast<float>(R.r14)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(((R.r9) ? (bitcast<float>(R.r14)) : ((0x0.0p+0f)))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r31) * static_cast<float>(bitcast<float>(R.r14))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(bitcast<float>(R.r14))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) * static_cast<float>(bitcast<float>(R.r14))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r25) * static_cast<float>(R.r36)));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r26) * static_cast<float>(R.r37)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r38)));
        R.r28 = static_cast<float>(static_cast<float>(static_cast<float>(R.r28) + static_cast<float>(R.r36)));
        R.r29 = static_cast<float>(static_cast<float>(static_cast<float>(R.r29) + static_cast<float>(R.r37)));
        R.r30 = static_cast<float>(static_cast<float>(static_cast<float>(R.r30) + static_cast<float>(R.r38)));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x6ull));
        if(R.r68) goto L_B45; else goto L_B1;
    L_B45: // direct_metal
        if(stop_heavy && !fresh) return 45;
    L_B45_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 45, 113u);
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r69) + static_cast<float>(bitcast<float>(R.r6))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r70) + static_cast<float>(bitcast<float>(R.r7))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r71) + static_cast<float>(R.r35)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r36, R.r36, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r37, R.r37, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, R.r38, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(bitcast<float>(R.r14))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) * static_cast<float>(bitcast<float>(R.r14))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>(bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>(R.r63))));
        R.r42 = static_cast<float>(op_fma(R.r66, R.r64, (-(bitcast<float>(R.r14)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(R.r64))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r62, (-(bitcast<float>(R.r14))))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>(R.r62))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r63, (-(bitcast<float>(R.r14))))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r36, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r66, R.r37, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r38, bitcast<float>(R.r14))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>(bitcast<float>(R.r14))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r36) - static_cast<float>(bitcast<float>(R.r48)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r37) - static_cast<float>(bitcast<float>(R.r49)))));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) - static_cast<float>(R.r50)));
        R.r52 = static_cast<float>((0x0.0p+0f));
        R.r52 = static_cast<float>(op_fma(bitcast<float>(R.r48), bitcast<float>(R.r48), R.r52));
        R.r52 = static_cast<float>(op_fma(bitcast<float>(R.r49), bitcast<float>(R.r49), R.r52));
        R.r52 = static_cast<float>(op_fma(R.r50, R.r50, R.r52));
        R.r52 = static_cast<float>(op_rsqrt(static_cast<float>(R.r52)));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) * static_cast<float>(R.r52))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) * static_cast<float>(R.r52))));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) * static_cast<float>(R.r52)));
        R.r51 = static_cast<float>((0x0.0p+0f));
        R.r51 = static_cast<float>(op_fma(bitcast<float>(R.r48), R.r62, R.r51));
        R.r51 = static_cast<float>(op_fma(bitcast<float>(R.r49), R.r63, R.r51));
        R.r51 = static_cast<float>(op_fma(R.r50, R.r64, R.r51));
        R.r52 = static_cast<float>((0x0.0p+0f));
        R.r52 = static_cast<float>(op_fma(bitcast<float>(R.r48), R.r42, R.r52));
        R.r52 = static_cast<float>(op_fma(bitcast<float>(R.r49), bitcast<float>(R.r43), R.r52));
        R.r52 = static_cast<float>(op_fma(R.r50, bitcast<float>(R.r44), R.r52));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r52)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) / static_cast<float>((0x1.9999980000000p-5f))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r51)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) / static_cast<float>((0x1.3333340000000p-2f))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) + static_cast<float>(R.r52)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(R.r51)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r14))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(R.r46)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) + static_cast<float>(R.r51)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) / static_cast<float>(R.r46)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>((0x1.4000000000000p+2f))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r14))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(R.r46)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r51)));
        R.r46 = static_cast<float>(op_fma(R.r46, R.r51, (0x1.0000000000000p+0f)));
        R.r46 = static_cast<float>(op_sqrt(static_cast<float>(R.r46)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) + static_cast<float>((0x1.0000000000000p+0f))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+1f)) / static_cast<float>(R.r46)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) * static_cast<float>(R.r46)));
        R.r52 = static_cast<float>((0x0.0p+0f));
        R.r52 = static_cast<float>(op_fma(R.r69, R.r62, R.r52));
        R.r52 = static_cast<float>(op_fma(R.r70, R.r63, R.r52));
        R.r52 = static_cast<float>(op_fma(R.r71, R.r64, R.r52));
        R.r36 = static_cast<float>((0x0.0p+0f));
        R.r36 = static_cast<float>(op_fma(R.r69, R.r42, R.r36));
        R.r36 = static_cast<float>(op_fma(R.r70, bitcast<float>(R.r43), R.r36));
        R.r36 = static_cast<float>(op_fma(R.r71, bitcast<float>(R.r44), R.r36));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(R.r36)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>((0x1.9999980000000p-5f))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>((0x1.9999980000000p-5f))));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r52)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>((0x1.3333340000000p-2f))));
        R.r52 = static_cast<float>(op_fma(R.r52, (0x1.3333340000000p-2f), R.r36));
        R.r52 = static_cast<float>(op_sqrt(static_cast<float>(R.r52)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r69, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r66, R.r70, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r71, bitcast<float>(R.r14))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r14))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(R.r46)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r52)));
        R.r46 = static_cast<float>(op_fma(R.r46, R.r52, (0x1.0000000000000p+0f)));
        R.r46 = static_cast<float>(op_sqrt(static_cast<float>(R.r46)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) + static_cast<float>((0x1.0000000000000p+0f))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+1f)) / static_cast<float>(R.r46)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) * static_cast<float>(R.r46)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>((0x1.0000000000000p+2f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r8)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>((0x1.0000000000000p-1f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_max<float>(static_cast<float>(bitcast<float>(R.r14)), static_cast<float>((0x1.47ae140000000p-7f)))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) / static_cast<float>(bitcast<float>(R.r14))));
        R.r45 = static_cast<float>(op_min<float>(static_cast<float>(R.r45), static_cast<float>((0x1.4000000000000p+2f))));
        R.r45 = static_cast<float>(((R.r9) ? (R.r45) : ((0x0.0p+0f))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r31) * static_cast<float>(R.r45)));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r32) * static_cast<float>(R.r45)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r33) * static_cast<float>(R.r45)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r25) * static_cast<float>(R.r36)));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r26) * static_cast<float>(R.r37)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r38)));
        R.r28 = static_cast<float>(static_cast<float>(static_cast<float>(R.r28) + static_cast<float>(R.r36)));
        R.r29 = static_cast<float>(static_cast<float>(static_cast<float>(R.r29) + static_cast<float>(R.r37)));
        R.r30 = static_cast<float>(static_cast<float>(static_cast<float>(R.r30) + static_cast<float>(R.r38)));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(-static_cast<float>(R.r69))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(-static_cast<float>(R.r70))));
        R.r35 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r71)));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x8ull));
        goto L_B1;
    L_B46: // window
        fresh = false;
        if constexpr(kProf) count_block(ctx, 46, 42u);
        R.r36 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r6))));
        R.r37 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r7))));
        R.r38 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r35)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r36, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r66, R.r37, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r38, bitcast<float>(R.r14))));
        R.r8 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) > static_cast<float>((0x0.0p+0f))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>((0x1.8f5c280000000p+0f))));
        R.r42 = static_cast<float>(((R.r8) ? (R.r42) : ((0x1.8f5c280000000p+0f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r14)))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r42))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) + static_cast<float>(R.r42)));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) / static_cast<float>(R.r51))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) * static_cast<float>(bitcast<float>(R.r48)))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r14))));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r51)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r52)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r51)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r48))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r52)));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) + static_cast<float>(R.r51))));
        R.r45 = static_cast<float>(bitcast<float>(R.r6));
        R.r46 = static_cast<float>(bitcast<float>(R.r7));
        R.r47 = static_cast<float>(R.r35);
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r14))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) + static_cast<float>(R.r45))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) + static_cast<float>(R.r46))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) + static_cast<float>(R.r47)));
        R.r43 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r20)) < static_cast<float>(bitcast<float>(R.r48))));
        R.r43 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r43) || static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r21)) < static_cast<float>((0x1.99999a0000000p-2f)))));
        R.r44 = static_cast<unsigned int>(op_min<unsigned int>(static_cast<unsigned int>(R.r43), static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r28 = static_cast<float>(((R.r43) ? (R.r28) : ((0x0.0p+0f))));
        R.r29 = static_cast<float>(((R.r43) ? (R.r29) : ((0x0.0p+0f))));
        R.r30 = static_cast<float>(((R.r43) ? (R.r30) : ((0x0.0p+0f))));
        if(R.r43) goto L_B4; else goto L_B53;
    L_B47: // lambert_indirect
        if(stop_heavy && !fresh) return 47;
    L_B47_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 47, 69u);
        R.r25 = static_cast<float>(static_cast<float>(static_cast<float>(R.r25) * static_cast<float>(R.r31)));
        R.r26 = static_cast<float>(static_cast<float>(static_cast<float>(R.r26) * static_cast<float>(R.r32)));
        R.r27 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r33)));
        R.r64 = static_cast<float>(op_copysign(static_cast<float>((0x1.0000000000000p+0f)), static_cast<float>(R.r67)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) + static_cast<float>(R.r67)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>((-0x1.0000000000000p+0f)) / static_cast<float>(R.r36)));
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(R.r66)));
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r62) * static_cast<float>(R.r36)));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(R.r66)));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r63) * static_cast<float>(R.r66)));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r63) + static_cast<float>(R.r64)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(R.r65)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(R.r65)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(R.r64)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) + static_cast<float>((0x1.0000000000000p+0f))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) * static_cast<float>(R.r62)));
        R.r38 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r64)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>(R.r65)));
        R.r64 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r66)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r36, R.r36, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r37, R.r37, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, R.r38, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(bitcast<float>(R.r14))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) * static_cast<float>(bitcast<float>(R.r14))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>(bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r62, R.r62, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r63, R.r63, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r64, R.r64, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r62) * static_cast<float>(bitcast<float>(R.r14))));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r63) * static_cast<float>(bitcast<float>(R.r14))));
        R.r64 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) * static_cast<float>(bitcast<float>(R.r14))));
        R.r20 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) - static_cast<float>((0x1.0000000000000p-1f)))));
        R.r20 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) * static_cast<float>((0x1.921fb60000000p+2f)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r21)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_cos(static_cast<float>(bitcast<float>(R.r20)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(bitcast<float>(R.r8))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) * static_cast<float>(bitcast<float>(R.r8))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>(bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_sin(static_cast<float>(bitcast<float>(R.r20)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r62) * static_cast<float>(bitcast<float>(R.r8))));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r63) * static_cast<float>(bitcast<float>(R.r8))));
        R.r64 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) * static_cast<float>(bitcast<float>(R.r8))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r21)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r65 = static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(bitcast<float>(R.r14))));
        R.r66 = static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>(bitcast<float>(R.r14))));
        R.r67 = static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>(bitcast<float>(R.r14))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r36) + static_cast<float>(R.r62))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r37) + static_cast<float>(R.r63))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) + static_cast<float>(R.r64)));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) + static_cast<float>(R.r65))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) + static_cast<float>(R.r66))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) + static_cast<float>(R.r67)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r35, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r14))));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x0ull));
        goto L_B4;
    L_B48: // tth_begin
        fresh = false;
        if constexpr(kProf) count_block(ctx, 48, 37u);
        R.r36 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r6))));
        R.r37 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r7))));
        R.r38 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r35)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r36, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r66, R.r37, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r38, bitcast<float>(R.r14))));
        R.r8 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) > static_cast<float>((0x0.0p+0f))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>((0x1.4000000000000p+1f))));
        R.r42 = static_cast<float>(((R.r8) ? (R.r42) : ((0x1.4000000000000p+1f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r14)))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r42))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) + static_cast<float>(R.r42)));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) / static_cast<float>(R.r51))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) * static_cast<float>(bitcast<float>(R.r48)))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r14))));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r51)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r52)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r51)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r48))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r52)));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) + static_cast<float>(R.r51))));
        R.r8 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r20)) < static_cast<float>(bitcast<float>(R.r48))));
        R.r45 = static_cast<float>(bitcast<float>(R.r6));
        R.r46 = static_cast<float>(bitcast<float>(R.r7));
        R.r47 = static_cast<float>(R.r35);
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r14))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) + static_cast<float>(R.r45))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) + static_cast<float>(R.r46))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) + static_cast<float>(R.r47)));
        R.r18 = static_cast<unsigned int>(((R.r8) ? (((unsigned int)0x0ull)) : (((unsigned int)0x1ull))));
        if(R.r8) goto L_B4; else goto L_B1;
    L_B49: // glass
        if(stop_heavy && !fresh) return 49;
    L_B49_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 49, 82u);
        R.r36 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r6))));
        R.r37 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r7))));
        R.r38 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r35)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r36, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r66, R.r37, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r38, bitcast<float>(R.r14))));
        R.r8 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r14)) > static_cast<float>((0x0.0p+0f))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>((0x1.8000000000000p+0f))));
        R.r42 = static_cast<float>(((R.r8) ? (R.r42) : ((0x1.8000000000000p+0f))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(bitcast<float>(R.r14)))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r42))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) + static_cast<float>(R.r42)));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) / static_cast<float>(R.r51))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) * static_cast<float>(bitcast<float>(R.r48)))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r14))));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r51)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r52)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r51)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r48))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r52)));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) + static_cast<float>(R.r51))));
        R.r54 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r65)));
        R.r55 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r66)));
        R.r56 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r67)));
        R.r65 = static_cast<float>(((R.r8) ? (R.r65) : (R.r54)));
        R.r66 = static_cast<float>(((R.r8) ? (R.r66) : (R.r55)));
        R.r67 = static_cast<float>(((R.r8) ? (R.r67) : (R.r56)));
        R.r9 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r6), R.r65, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r7), R.r66, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r35, R.r67, bitcast<float>(R.r9))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r9)) * static_cast<float>(bitcast<float>(R.r9)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r8)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r42) * static_cast<float>(bitcast<float>(R.r8)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r42) * static_cast<float>(bitcast<float>(R.r8)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r8)))));
        R.r45 = static_cast<float>(bitcast<float>(R.r6));
        R.r46 = static_cast<float>(bitcast<float>(R.r7));
        R.r47 = static_cast<float>(R.r35);
        R.r54 = static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r8))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r9), R.r42, R.r54)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(bitcast<float>(R.r9))));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>(bitcast<float>(R.r9))));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>(bitcast<float>(R.r9)))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r42))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r42))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(R.r42)));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) - static_cast<float>(R.r51))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) - static_cast<float>(R.r52))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) - static_cast<float>(bitcast<float>(R.r53))));
        R.r54 = static_cast<float>((0x0.0p+0f));
        R.r54 = static_cast<float>(op_fma(bitcast<float>(R.r6), bitcast<float>(R.r6), R.r54));
        R.r54 = static_cast<float>(op_fma(bitcast<float>(R.r7), bitcast<float>(R.r7), R.r54));
        R.r54 = static_cast<float>(op_fma(R.r35, R.r35, R.r54));
        R.r54 = static_cast<float>(op_rsqrt(static_cast<float>(R.r54)));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(R.r54))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(R.r54))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(R.r54)));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r54) * static_cast<float>(bitcast<float>(R.r14))));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r55) * static_cast<float>(bitcast<float>(R.r14))));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r56) * static_cast<float>(bitcast<float>(R.r14))));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r54) + static_cast<float>(R.r45)));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r55) + static_cast<float>(R.r46)));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r56) + static_cast<float>(R.r47)));
        R.r14 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r8)) < static_cast<float>((0x0.0p+0f))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r14) || static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r20)) < static_cast<float>(bitcast<float>(R.r48)))));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) * static_cast<float>(R.r42)));
        R.r31 = static_cast<float>(static_cast<float>(static_cast<float>(R.r25) / static_cast<float>(R.r42)));
        R.r32 = static_cast<float>(static_cast<float>(static_cast<float>(R.r26) / static_cast<float>(R.r42)));
        R.r33 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) / static_cast<float>(R.r42)));
        R.r6 = bitcast<unsigned int>(static_cast<float>(((R.r14) ? (R.r54) : (bitcast<float>(R.r6)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(((R.r14) ? (R.r55) : (bitcast<float>(R.r7)))));
        R.r35 = static_cast<float>(((R.r14) ? (R.r56) : (R.r35)));
        R.r25 = static_cast<float>(((R.r14) ? (R.r25) : (R.r31)));
        R.r26 = static_cast<float>(((R.r14) ? (R.r26) : (R.r32)));
        R.r27 = static_cast<float>(((R.r14) ? (R.r27) : (R.r33)));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x0ull));
        goto L_B4;
    L_B50: // indirect_metal
        fresh = false;
        if constexpr(kProf) count_block(ctx, 50, 27u);
        R.r25 = static_cast<float>(static_cast<float>(static_cast<float>(R.r25) * static_cast<float>(R.r31)));
        R.r26 = static_cast<float>(static_cast<float>(static_cast<float>(R.r26) * static_cast<float>(R.r32)));
        R.r27 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r33)));
        R.r36 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r6))));
        R.r37 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r7))));
        R.r38 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r35)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>((0x1.3333340000000p-2f))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) * static_cast<float>((0x1.9999980000000p-5f))));
        R.r9 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r36, R.r36, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r37, R.r37, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r38, R.r38, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r9)))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(bitcast<float>(R.r9))));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) * static_cast<float>(bitcast<float>(R.r9))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>(bitcast<float>(R.r9))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r20)))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) / static_cast<float>(bitcast<float>(R.r48)))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r48)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(bitcast<float>(R.r21)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.921fb60000000p+2f)) * static_cast<float>(bitcast<float>(R.r49)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_cos(static_cast<float>(bitcast<float>(R.r49)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r48)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_sin(static_cast<float>(bitcast<float>(R.r49)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) * static_cast<float>(bitcast<float>(R.r48)))));
        R.r9 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r38) > static_cast<float>((0x1.fff2e40000000p-1f))));
        if(R.r9) goto L_B52; else goto L_B51;
    L_B51: // get_slope_mid
        if(stop_heavy && !fresh) return 51;
    L_B51_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 51, 53u);
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>(R.r38)));
        R.r9 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r38))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_max<float>(static_cast<float>(R.r38), static_cast<float>((0x1.0c6f7a0000000p-20f)))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r9)) / static_cast<float>(bitcast<float>(R.r49)))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r9)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(bitcast<float>(R.r48)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) * static_cast<float>(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) + static_cast<float>(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) + static_cast<float>(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+1f)) / static_cast<float>(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r20)) / static_cast<float>(bitcast<float>(R.r49)))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r49), (0x1.0000000000000p+1f), (-((0x1.0000000000000p+0f))))));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) * static_cast<float>(bitcast<float>(R.r49))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r52 = static_cast<float>(op_copysign(static_cast<float>((0x1.0c6f7a0000000p-20f)), static_cast<float>(R.r51)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(op_abs(static_cast<float>(R.r51))));
        R.r53 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r53)) < static_cast<float>((0x1.0c6f7a0000000p-20f))));
        R.r51 = static_cast<float>(((R.r53) ? (R.r52) : (R.r51)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(R.r51)));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) - static_cast<float>(bitcast<float>(R.r9))));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) * static_cast<float>(R.r51)));
        R.r9 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r9)) * static_cast<float>(R.r51))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r9), R.r51, (-(R.r50)))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r9)))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) * static_cast<float>(R.r51)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r51) - static_cast<float>(bitcast<float>(R.r9)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r51) + static_cast<float>(bitcast<float>(R.r9)))));
        R.r49 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r49)) < static_cast<float>((0x0.0p+0f))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(bitcast<float>(R.r48)))));
        R.r49 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r49) || static_cast<unsigned int>(static_cast<float>(bitcast<float>(R.r8)) > static_cast<float>(bitcast<float>(R.r48)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(((R.r49) ? (bitcast<float>(R.r14)) : (bitcast<float>(R.r8)))));
        R.r48 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r21)) > static_cast<float>((0x1.0000000000000p-1f))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r21)) - static_cast<float>((0x1.0000000000000p-1f)))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r9)) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r21 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p-1f)) - static_cast<float>(bitcast<float>(R.r21)))));
        R.r21 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r21)) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r21 = bitcast<unsigned int>(static_cast<float>(((R.r48) ? (bitcast<float>(R.r9)) : (bitcast<float>(R.r21)))));
        R.r20 = bitcast<unsigned int>(static_cast<float>(((R.r48) ? ((0x1.0000000000000p+0f)) : ((-0x1.0000000000000p+0f)))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r21), (0x1.7d3a1e0000000p-4f), (0x1.3cd8980000000p-2f))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r9), bitcast<float>(R.r21), (-0x1.0000000000000p+0f))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r9), bitcast<float>(R.r21), (0x1.322cec0000000p-1f))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r21), (0x1.186c220000000p-2f), (-0x1.77a6360000000p-1f))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(op_fma(bitcast<float>(R.r48), bitcast<float>(R.r21), (0x1.da88260000000p-2f))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) * static_cast<float>(bitcast<float>(R.r21)))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) / static_cast<float>(bitcast<float>(R.r9)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) + static_cast<float>((0x1.0000000000000p+0f)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r8)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) * static_cast<float>(bitcast<float>(R.r48)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) * static_cast<float>(bitcast<float>(R.r20)))));
        goto L_B52;
    L_B52: // get_slope_end
        if(stop_heavy && !fresh) return 52;
    L_B52_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 52, 128u);
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r37) * static_cast<float>(R.r37))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r36, R.r36, bitcast<float>(R.r48))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r9)))));
        R.r48 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r9)) > static_cast<float>((0x1.1979980000000p-40f))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r36) / static_cast<float>(bitcast<float>(R.r9)))));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r37) / static_cast<float>(bitcast<float>(R.r9))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(((R.r48) ? (bitcast<float>(R.r49)) : ((0x1.0000000000000p+0f)))));
        R.r50 = static_cast<float>(((R.r48) ? (R.r50) : ((0x0.0p+0f))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) * static_cast<float>(bitcast<float>(R.r14))));
        R.r45 = static_cast<float>(op_fma(R.r50, bitcast<float>(R.r8), R.r45));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) * static_cast<float>((0x1.3333340000000p-2f))));
        R.r50 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r50)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) * static_cast<float>(bitcast<float>(R.r14))));
        R.r46 = static_cast<float>(op_fma(bitcast<float>(R.r49), bitcast<float>(R.r8), R.r46));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>((0x1.9999980000000p-5f))));
        R.r47 = static_cast<float>((0x1.0000000000000p+0f));
        R.r45 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r45)));
        R.r46 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r46)));
        R.r9 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r45, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, R.r46, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, R.r47, bitcast<float>(R.r9))));
        R.r9 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r9)))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) * static_cast<float>(bitcast<float>(R.r9))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>(bitcast<float>(R.r9))));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) * static_cast<float>(bitcast<float>(R.r9))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>(R.r63))));
        R.r42 = static_cast<float>(op_fma(R.r66, R.r64, (-(bitcast<float>(R.r14)))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(R.r64))));
        R.r43 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r62, (-(bitcast<float>(R.r14))))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>(R.r62))));
        R.r44 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r63, (-(bitcast<float>(R.r14))))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r62) * static_cast<float>(R.r45))));
        R.r49 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r63) * static_cast<float>(R.r45))));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) * static_cast<float>(R.r45)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) * static_cast<float>(R.r46)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r43)) * static_cast<float>(R.r46)));
        R.r53 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r44)) * static_cast<float>(R.r46))));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(R.r47)));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>(R.r47)));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>(R.r47)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r48)) + static_cast<float>(R.r51)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r49)) + static_cast<float>(R.r52)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) + static_cast<float>(bitcast<float>(R.r53))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) + static_cast<float>(R.r54)));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) + static_cast<float>(R.r55)));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) + static_cast<float>(R.r56)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r45, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, R.r46, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, R.r47, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_rsqrt(static_cast<float>(bitcast<float>(R.r14)))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) * static_cast<float>(bitcast<float>(R.r14))));
        R.r46 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>(bitcast<float>(R.r14))));
        R.r47 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) * static_cast<float>(bitcast<float>(R.r14))));
        R.r36 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r6))));
        R.r37 = static_cast<float>(static_cast<float>(-static_cast<float>(bitcast<float>(R.r7))));
        R.r38 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r35)));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r45, R.r36, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r46, R.r37, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r47, R.r38, bitcast<float>(R.r14))));
        R.r48 = bitcast<unsigned int>(static_cast<float>(bitcast<float>(R.r6)));
        R.r49 = bitcast<unsigned int>(static_cast<float>(bitcast<float>(R.r7)));
        R.r50 = static_cast<float>(R.r35);
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r45) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r46) * static_cast<float>((0x1.0000000000000p+1f)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) * static_cast<float>(bitcast<float>(R.r14)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) * static_cast<float>(bitcast<float>(R.r14))));
        R.r6 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r6)) + static_cast<float>(bitcast<float>(R.r48)))));
        R.r7 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r7)) + static_cast<float>(bitcast<float>(R.r49)))));
        R.r35 = static_cast<float>(static_cast<float>(static_cast<float>(R.r35) + static_cast<float>(R.r50)));
        R.r8 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, bitcast<float>(R.r6), bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r66, bitcast<float>(R.r7), bitcast<float>(R.r8))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r35, bitcast<float>(R.r8))));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r65, R.r45, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r66, R.r46, bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r67, R.r47, bitcast<float>(R.r14))));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r65) * static_cast<float>(bitcast<float>(R.r14))));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r66) * static_cast<float>(bitcast<float>(R.r14))));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r67) * static_cast<float>(bitcast<float>(R.r14))));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r45) - static_cast<float>(R.r54)));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r46) - static_cast<float>(R.r55)));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r47) - static_cast<float>(R.r56)));
        R.r52 = static_cast<float>((0x0.0p+0f));
        R.r52 = static_cast<float>(op_fma(R.r54, R.r54, R.r52));
        R.r52 = static_cast<float>(op_fma(R.r55, R.r55, R.r52));
        R.r52 = static_cast<float>(op_fma(R.r56, R.r56, R.r52));
        R.r52 = static_cast<float>(op_rsqrt(static_cast<float>(R.r52)));
        R.r54 = static_cast<float>(static_cast<float>(static_cast<float>(R.r54) * static_cast<float>(R.r52)));
        R.r55 = static_cast<float>(static_cast<float>(static_cast<float>(R.r55) * static_cast<float>(R.r52)));
        R.r56 = static_cast<float>(static_cast<float>(static_cast<float>(R.r56) * static_cast<float>(R.r52)));
        R.r51 = static_cast<float>((0x0.0p+0f));
        R.r51 = static_cast<float>(op_fma(R.r54, R.r62, R.r51));
        R.r51 = static_cast<float>(op_fma(R.r55, R.r63, R.r51));
        R.r51 = static_cast<float>(op_fma(R.r56, R.r64, R.r51));
        R.r52 = static_cast<float>((0x0.0p+0f));
        R.r52 = static_cast<float>(op_fma(R.r54, R.r42, R.r52));
        R.r52 = static_cast<float>(op_fma(R.r55, bitcast<float>(R.r43), R.r52));
        R.r52 = static_cast<float>(op_fma(R.r56, bitcast<float>(R.r44), R.r52));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) * static_cast<float>(R.r52)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) / static_cast<float>((0x1.9999980000000p-5f))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r51)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) / static_cast<float>((0x1.3333340000000p-2f))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) + static_cast<float>(R.r52)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(R.r51)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) * static_cast<float>(bitcast<float>(R.r14))));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>(R.r52)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r51)));
        R.r52 = static_cast<float>(op_fma(R.r52, R.r51, (0x1.0000000000000p+0f)));
        R.r52 = static_cast<float>(op_sqrt(static_cast<float>(R.r52)));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>(R.r52) + static_cast<float>((0x1.0000000000000p+0f))));
        R.r52 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+1f)) / static_cast<float>(R.r52)));
        R.r52 = static_cast<float>(op_max<float>(static_cast<float>(R.r52), static_cast<float>((0x1.0624de0000000p-10f))));
        R.r25 = static_cast<float>(static_cast<float>(static_cast<float>(R.r25) * static_cast<float>(R.r52)));
        R.r26 = static_cast<float>(static_cast<float>(static_cast<float>(R.r26) * static_cast<float>(R.r52)));
        R.r27 = static_cast<float>(static_cast<float>(static_cast<float>(R.r27) * static_cast<float>(R.r52)));
        R.r9 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r8)) < static_cast<float>((0x0.0p+0f))));
        R.r25 = static_cast<float>(((R.r9) ? ((0x0.0p+0f)) : (R.r25)));
        R.r26 = static_cast<float>(((R.r9) ? ((0x0.0p+0f)) : (R.r26)));
        R.r27 = static_cast<float>(((R.r9) ? ((0x0.0p+0f)) : (R.r27)));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x0ull));
        if(R.r9) goto L_B53; else goto L_B4;
    L_B53: // fin_sample
        fresh = false;
        if constexpr(kProf) count_block(ctx, 53, 23u);
        R.r2 = static_cast<float>(static_cast<float>(static_cast<float>(R.r2) + static_cast<float>(R.r28)));
        R.r3 = static_cast<float>(static_cast<float>(static_cast<float>(R.r3) + static_cast<float>(R.r29)));
        R.r4 = static_cast<float>(static_cast<float>(static_cast<float>(R.r4) + static_cast<float>(R.r30)));
        R.r9 = bitcast<unsigned int>(static_cast<float>(R.r19));
        R.r14 = bitcast<unsigned int>(static_cast<float>((0x0.0p+0f)));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r28, (0x1.b367a00000000p-3f), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r29, (0x1.6e2eb20000000p-1f), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_fma(R.r30, (0x1.27bb300000000p-4f), bitcast<float>(R.r14))));
        R.r14 = bitcast<unsigned int>(static_cast<float>(op_min<float>(static_cast<float>(bitcast<float>(R.r14)), static_cast<float>((0x1.0000000000000p+0f)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) - static_cast<float>(R.r16))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) / static_cast<float>(bitcast<float>(R.r9))));
        R.r16 = static_cast<float>(static_cast<float>(static_cast<float>(R.r16) + static_cast<float>(R.r36)));
        R.r37 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r14)) - static_cast<float>(R.r16)));
        R.r17 = static_cast<float>(op_fma(bitcast<float>(R.r8), R.r37, R.r17));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) - static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(R.r8));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(R.r17) / static_cast<float>(bitcast<float>(R.r8)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(op_sqrt(static_cast<float>(bitcast<float>(R.r8)))));
        R.r8 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r8)) / static_cast<float>(bitcast<float>(R.r9)))));
        R.r8 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r8)) < static_cast<float>((0x1.0624de0000000p-10f))));
        R.r14 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r8) && static_cast<unsigned int>(static_cast<unsigned int>(R.r19) >= static_cast<unsigned int>(((unsigned int)0x40ull)))));
        R.r18 = static_cast<unsigned int>(((unsigned int)0x0ull));
        if(R.r14) goto L_B54; else goto L_B1;
    L_B54: // fin_pixel
        fresh = false;
        if constexpr(kProf) count_block(ctx, 54, 5u);
        R.r19 = bitcast<unsigned int>(static_cast<float>(R.r19));
        R.r2 = static_cast<float>(static_cast<float>(static_cast<float>(R.r2) / static_cast<float>(bitcast<float>(R.r19))));
        R.r3 = static_cast<float>(static_cast<float>(static_cast<float>(R.r3) / static_cast<float>(bitcast<float>(R.r19))));
        R.r4 = static_cast<float>(static_cast<float>(static_cast<float>(R.r4) / static_cast<float>(bitcast<float>(R.r19))));
        goto L_HALT;
    L_HALT:
        return kHalt;
    }

    static constexpr unsigned long long kRowBytes = 10032ull;
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
                v0.y = bitcast<unsigned>(R.r14);
                v0.z = bitcast<unsigned>(R.r22);
                v0.w = bitcast<unsigned>(R.r23);
                reinterpret_cast<uint4*>(base + 0ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r24);
                v1.y = bitcast<unsigned>(R.r25);
                v1.z = bitcast<unsigned>(R.r26);
                v1.w = bitcast<unsigned>(R.r27);
                reinterpret_cast<uint4*>(base + 16ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r28);
                v2.y = bitcast<unsigned>(R.r29);
                v2.z = bitcast<unsigned>(R.r30);
                v2.w = bitcast<unsigned>(R.r31);
                reinterpret_cast<uint4*>(base + 32ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r32);
                v3.y = bitcast<unsigned>(R.r33);
                v3.z = bitcast<unsigned>(R.r34);
                v3.w = bitcast<unsigned>(R.r35);
                reinterpret_cast<uint4*>(base + 48ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r61);
                v4.y = bitcast<unsigned>(R.r62);
                v4.z = bitcast<unsigned>(R.r63);
                v4.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 64ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r65);
                v5.y = bitcast<unsigned>(R.r66);
                v5.z = bitcast<unsigned>(R.r67);
                v5.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 80ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r69);
                v6.y = bitcast<unsigned>(R.r70);
                v6.z = bitcast<unsigned>(R.r71);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 96ull * cap)[idx] = v6;
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
                reinterpret_cast<uint4*>(base + 112ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 128ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 144ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 160ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 176ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 192ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 208ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 224ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r65);
                v8.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 240ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r67);
                v9.y = bitcast<unsigned>(R.r68);
                v9.z = bitcast<unsigned>(R.r69);
                v9.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 256ull * cap)[idx] = v9;
            }
            {
                uint2 v10;
                v10.x = bitcast<unsigned>(R.r71);
                v10.y = tid;
                reinterpret_cast<uint2*>(base + 272ull * cap)[idx] = v10;
            }
            return;
        }
        case 2: // roll_split
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
                v2.y = bitcast<unsigned>(R.r10);
                v2.z = bitcast<unsigned>(R.r11);
                v2.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 312ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r13);
                v3.y = bitcast<unsigned>(R.r15);
                v3.z = bitcast<unsigned>(R.r16);
                v3.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 328ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r18);
                v4.y = bitcast<unsigned>(R.r19);
                v4.z = bitcast<unsigned>(R.r20);
                v4.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 344ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r22);
                v5.y = bitcast<unsigned>(R.r23);
                v5.z = bitcast<unsigned>(R.r24);
                v5.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 360ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r26);
                v6.y = bitcast<unsigned>(R.r27);
                v6.z = bitcast<unsigned>(R.r28);
                v6.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 376ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r30);
                v7.y = bitcast<unsigned>(R.r31);
                v7.z = bitcast<unsigned>(R.r32);
                v7.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 392ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r34);
                v8.y = bitcast<unsigned>(R.r35);
                v8.z = bitcast<unsigned>(R.r61);
                v8.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 408ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r63);
                v9.y = bitcast<unsigned>(R.r64);
                v9.z = bitcast<unsigned>(R.r65);
                v9.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 424ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r67);
                v10.y = bitcast<unsigned>(R.r68);
                v10.z = bitcast<unsigned>(R.r69);
                v10.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 440ull * cap)[idx] = v10;
            }
            {
                uint2 v11;
                v11.x = bitcast<unsigned>(R.r71);
                v11.y = tid;
                reinterpret_cast<uint2*>(base + 456ull * cap)[idx] = v11;
            }
            return;
        }
        case 3: // sample_pixel
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 464ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r10);
                v1.z = bitcast<unsigned>(R.r11);
                v1.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 480ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r13);
                v2.y = bitcast<unsigned>(R.r15);
                v2.z = bitcast<unsigned>(R.r16);
                v2.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 496ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r18);
                v3.y = bitcast<unsigned>(R.r19);
                v3.z = bitcast<unsigned>(R.r20);
                v3.w = bitcast<unsigned>(R.r21);
                reinterpret_cast<uint4*>(base + 512ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r61);
                v4.y = bitcast<unsigned>(R.r62);
                v4.z = bitcast<unsigned>(R.r63);
                v4.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 528ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r65);
                v5.y = bitcast<unsigned>(R.r66);
                v5.z = bitcast<unsigned>(R.r67);
                v5.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 544ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r69);
                v6.y = bitcast<unsigned>(R.r70);
                v6.z = bitcast<unsigned>(R.r71);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 560ull * cap)[idx] = v6;
            }
            return;
        }
        case 4: // traverse_scene
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 576ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 592ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 608ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 624ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 640ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 656ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 672ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 688ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r65);
                v8.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 704ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r67);
                v9.y = bitcast<unsigned>(R.r68);
                v9.z = bitcast<unsigned>(R.r69);
                v9.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 720ull * cap)[idx] = v9;
            }
            {
                uint2 v10;
                v10.x = bitcast<unsigned>(R.r71);
                v10.y = tid;
                reinterpret_cast<uint2*>(base + 736ull * cap)[idx] = v10;
            }
            return;
        }
        case 5: // traverse_box
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
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 760ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 776ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 792ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 808ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 824ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 840ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 856ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r61);
                v8.z = bitcast<unsigned>(R.r62);
                v8.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 872ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r64);
                v9.y = bitcast<unsigned>(R.r65);
                v9.z = bitcast<unsigned>(R.r66);
                v9.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 888ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r68);
                v10.y = bitcast<unsigned>(R.r69);
                v10.z = bitcast<unsigned>(R.r70);
                v10.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 904ull * cap)[idx] = v10;
            }
            {
                unsigned v11;
                v11 = tid;
                reinterpret_cast<unsigned*>(base + 920ull * cap)[idx] = v11;
            }
            return;
        }
        case 6: // isect_quad_l1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 928ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 944ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 960ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 976ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 992ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 1008ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 1024ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 1040ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r39);
                v8.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 1056ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r41);
                v9.y = bitcast<unsigned>(R.r42);
                v9.z = bitcast<unsigned>(R.r43);
                v9.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 1072ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r45);
                v10.y = bitcast<unsigned>(R.r46);
                v10.z = bitcast<unsigned>(R.r47);
                v10.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 1088ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r49);
                v11.y = bitcast<unsigned>(R.r50);
                v11.z = bitcast<unsigned>(R.r58);
                v11.w = bitcast<unsigned>(R.r59);
                reinterpret_cast<uint4*>(base + 1104ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r60);
                v12.y = bitcast<unsigned>(R.r61);
                v12.z = bitcast<unsigned>(R.r62);
                v12.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 1120ull * cap)[idx] = v12;
            }
            {
                uint4 v13;
                v13.x = bitcast<unsigned>(R.r64);
                v13.y = bitcast<unsigned>(R.r65);
                v13.z = bitcast<unsigned>(R.r66);
                v13.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 1136ull * cap)[idx] = v13;
            }
            {
                uint4 v14;
                v14.x = bitcast<unsigned>(R.r68);
                v14.y = bitcast<unsigned>(R.r69);
                v14.z = bitcast<unsigned>(R.r70);
                v14.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 1152ull * cap)[idx] = v14;
            }
            {
                unsigned v15;
                v15 = tid;
                reinterpret_cast<unsigned*>(base + 1168ull * cap)[idx] = v15;
            }
            return;
        }
        case 7: // isect_quad_l2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1176ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1192ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r10);
                v2.y = bitcast<unsigned>(R.r11);
                v2.z = bitcast<unsigned>(R.r12);
                v2.w = bitcast<unsigned>(R.r13);
                reinterpret_cast<uint4*>(base + 1208ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r14);
                v3.y = bitcast<unsigned>(R.r15);
                v3.z = bitcast<unsigned>(R.r16);
                v3.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 1224ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r18);
                v4.y = bitcast<unsigned>(R.r19);
                v4.z = bitcast<unsigned>(R.r22);
                v4.w = bitcast<unsigned>(R.r23);
                reinterpret_cast<uint4*>(base + 1240ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r24);
                v5.y = bitcast<unsigned>(R.r25);
                v5.z = bitcast<unsigned>(R.r26);
                v5.w = bitcast<unsigned>(R.r27);
                reinterpret_cast<uint4*>(base + 1256ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r28);
                v6.y = bitcast<unsigned>(R.r29);
                v6.z = bitcast<unsigned>(R.r30);
                v6.w = bitcast<unsigned>(R.r31);
                reinterpret_cast<uint4*>(base + 1272ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r32);
                v7.y = bitcast<unsigned>(R.r33);
                v7.z = bitcast<unsigned>(R.r34);
                v7.w = bitcast<unsigned>(R.r35);
                reinterpret_cast<uint4*>(base + 1288ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r36);
                v8.y = bitcast<unsigned>(R.r37);
                v8.z = bitcast<unsigned>(R.r38);
                v8.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 1304ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r40);
                v9.y = bitcast<unsigned>(R.r41);
                v9.z = bitcast<unsigned>(R.r42);
                v9.w = bitcast<unsigned>(R.r43);
                reinterpret_cast<uint4*>(base + 1320ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r44);
                v10.y = bitcast<unsigned>(R.r45);
                v10.z = bitcast<unsigned>(R.r46);
                v10.w = bitcast<unsigned>(R.r47);
                reinterpret_cast<uint4*>(base + 1336ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r48);
                v11.y = bitcast<unsigned>(R.r49);
                v11.z = bitcast<unsigned>(R.r50);
                v11.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 1352ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r62);
                v12.y = bitcast<unsigned>(R.r63);
                v12.z = bitcast<unsigned>(R.r64);
                v12.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 1368ull * cap)[idx] = v12;
            }
            {
                uint4 v13;
                v13.x = bitcast<unsigned>(R.r66);
                v13.y = bitcast<unsigned>(R.r67);
                v13.z = bitcast<unsigned>(R.r68);
                v13.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 1384ull * cap)[idx] = v13;
            }
            {
                uint4 v14;
                v14.x = bitcast<unsigned>(R.r70);
                v14.y = bitcast<unsigned>(R.r71);
                v14.z = tid;
                reinterpret_cast<uint4*>(base + 1400ull * cap)[idx] = v14;
            }
            return;
        }
        case 8: // isect_quad_l3
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1416ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 1432ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r10);
                v2.z = bitcast<unsigned>(R.r11);
                v2.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 1448ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r13);
                v3.y = bitcast<unsigned>(R.r14);
                v3.z = bitcast<unsigned>(R.r15);
                v3.w = bitcast<unsigned>(R.r16);
                reinterpret_cast<uint4*>(base + 1464ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r17);
                v4.y = bitcast<unsigned>(R.r18);
                v4.z = bitcast<unsigned>(R.r19);
                v4.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 1480ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r23);
                v5.y = bitcast<unsigned>(R.r24);
                v5.z = bitcast<unsigned>(R.r25);
                v5.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 1496ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r27);
                v6.y = bitcast<unsigned>(R.r28);
                v6.z = bitcast<unsigned>(R.r29);
                v6.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 1512ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r31);
                v7.y = bitcast<unsigned>(R.r32);
                v7.z = bitcast<unsigned>(R.r33);
                v7.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 1528ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r35);
                v8.y = bitcast<unsigned>(R.r36);
                v8.z = bitcast<unsigned>(R.r37);
                v8.w = bitcast<unsigned>(R.r38);
                reinterpret_cast<uint4*>(base + 1544ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r39);
                v9.y = bitcast<unsigned>(R.r40);
                v9.z = bitcast<unsigned>(R.r41);
                v9.w = bitcast<unsigned>(R.r42);
                reinterpret_cast<uint4*>(base + 1560ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r43);
                v10.y = bitcast<unsigned>(R.r44);
                v10.z = bitcast<unsigned>(R.r45);
                v10.w = bitcast<unsigned>(R.r46);
                reinterpret_cast<uint4*>(base + 1576ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r47);
                v11.y = bitcast<unsigned>(R.r48);
                v11.z = bitcast<unsigned>(R.r49);
                v11.w = bitcast<unsigned>(R.r50);
                reinterpret_cast<uint4*>(base + 1592ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r62);
                v12.y = bitcast<unsigned>(R.r63);
                v12.z = bitcast<unsigned>(R.r64);
                v12.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 1608ull * cap)[idx] = v12;
            }
            {
                uint4 v13;
                v13.x = bitcast<unsigned>(R.r66);
                v13.y = bitcast<unsigned>(R.r67);
                v13.z = bitcast<unsigned>(R.r68);
                v13.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 1624ull * cap)[idx] = v13;
            }
            {
                uint4 v14;
                v14.x = bitcast<unsigned>(R.r70);
                v14.y = bitcast<unsigned>(R.r71);
                v14.z = tid;
                reinterpret_cast<uint4*>(base + 1640ull * cap)[idx] = v14;
            }
            return;
        }
        case 9: // isect_quad_l4
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1656ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 1672ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 1688ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 1704ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1720ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 1736ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 1752ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 1768ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r39);
                v8.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 1784ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r41);
                v9.y = bitcast<unsigned>(R.r42);
                v9.z = bitcast<unsigned>(R.r43);
                v9.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 1800ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r45);
                v10.y = bitcast<unsigned>(R.r46);
                v10.z = bitcast<unsigned>(R.r47);
                v10.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 1816ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r49);
                v11.y = bitcast<unsigned>(R.r50);
                v11.z = bitcast<unsigned>(R.r62);
                v11.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 1832ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r64);
                v12.y = bitcast<unsigned>(R.r65);
                v12.z = bitcast<unsigned>(R.r66);
                v12.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 1848ull * cap)[idx] = v12;
            }
            {
                uint4 v13;
                v13.x = bitcast<unsigned>(R.r68);
                v13.y = bitcast<unsigned>(R.r69);
                v13.z = bitcast<unsigned>(R.r70);
                v13.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 1864ull * cap)[idx] = v13;
            }
            {
                unsigned v14;
                v14 = tid;
                reinterpret_cast<unsigned*>(base + 1880ull * cap)[idx] = v14;
            }
            return;
        }
        case 10: // isect_quad_l5
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 1888ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 1904ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 1920ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 1936ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1952ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 1968ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 1984ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 2000ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r39);
                v8.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 2016ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r41);
                v9.y = bitcast<unsigned>(R.r42);
                v9.z = bitcast<unsigned>(R.r43);
                v9.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 2032ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r45);
                v10.y = bitcast<unsigned>(R.r46);
                v10.z = bitcast<unsigned>(R.r47);
                v10.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 2048ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r49);
                v11.y = bitcast<unsigned>(R.r50);
                v11.z = bitcast<unsigned>(R.r51);
                v11.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 2064ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r53);
                v12.y = bitcast<unsigned>(R.r58);
                v12.z = bitcast<unsigned>(R.r59);
                v12.w = bitcast<unsigned>(R.r60);
                reinterpret_cast<uint4*>(base + 2080ull * cap)[idx] = v12;
            }
            {
                uint4 v13;
                v13.x = bitcast<unsigned>(R.r61);
                v13.y = bitcast<unsigned>(R.r62);
                v13.z = bitcast<unsigned>(R.r63);
                v13.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 2096ull * cap)[idx] = v13;
            }
            {
                uint4 v14;
                v14.x = bitcast<unsigned>(R.r65);
                v14.y = bitcast<unsigned>(R.r66);
                v14.z = bitcast<unsigned>(R.r67);
                v14.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 2112ull * cap)[idx] = v14;
            }
            {
                uint4 v15;
                v15.x = bitcast<unsigned>(R.r69);
                v15.y = bitcast<unsigned>(R.r70);
                v15.z = bitcast<unsigned>(R.r71);
                v15.w = tid;
                reinterpret_cast<uint4*>(base + 2128ull * cap)[idx] = v15;
            }
            return;
        }
        case 11: // isect_quad_l6
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2144ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 2160ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 2176ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 2192ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 2208ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 2224ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 2240ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 2256ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r39);
                v8.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 2272ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r41);
                v9.y = bitcast<unsigned>(R.r42);
                v9.z = bitcast<unsigned>(R.r43);
                v9.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 2288ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r48);
                v10.y = bitcast<unsigned>(R.r49);
                v10.z = bitcast<unsigned>(R.r50);
                v10.w = bitcast<unsigned>(R.r51);
                reinterpret_cast<uint4*>(base + 2304ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r52);
                v11.y = bitcast<unsigned>(R.r53);
                v11.z = bitcast<unsigned>(R.r54);
                v11.w = bitcast<unsigned>(R.r55);
                reinterpret_cast<uint4*>(base + 2320ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r56);
                v12.y = bitcast<unsigned>(R.r61);
                v12.z = bitcast<unsigned>(R.r62);
                v12.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 2336ull * cap)[idx] = v12;
            }
            {
                uint4 v13;
                v13.x = bitcast<unsigned>(R.r64);
                v13.y = bitcast<unsigned>(R.r65);
                v13.z = bitcast<unsigned>(R.r66);
                v13.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 2352ull * cap)[idx] = v13;
            }
            {
                uint4 v14;
                v14.x = bitcast<unsigned>(R.r68);
                v14.y = bitcast<unsigned>(R.r69);
                v14.z = bitcast<unsigned>(R.r70);
                v14.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 2368ull * cap)[idx] = v14;
            }
            {
                unsigned v15;
                v15 = tid;
                reinterpret_cast<unsigned*>(base + 2384ull * cap)[idx] = v15;
            }
            return;
        }
        case 12: // isect_quad_l7
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2392ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 2408ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 2424ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 2440ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 2456ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 2472ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 2488ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 2504ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r39);
                v8.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 2520ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r41);
                v9.y = bitcast<unsigned>(R.r42);
                v9.z = bitcast<unsigned>(R.r43);
                v9.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 2536ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r48);
                v10.y = bitcast<unsigned>(R.r49);
                v10.z = bitcast<unsigned>(R.r50);
                v10.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 2552ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r63);
                v11.y = bitcast<unsigned>(R.r64);
                v11.z = bitcast<unsigned>(R.r65);
                v11.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 2568ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r67);
                v12.y = bitcast<unsigned>(R.r68);
                v12.z = bitcast<unsigned>(R.r69);
                v12.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 2584ull * cap)[idx] = v12;
            }
            {
                uint2 v13;
                v13.x = bitcast<unsigned>(R.r71);
                v13.y = tid;
                reinterpret_cast<uint2*>(base + 2600ull * cap)[idx] = v13;
            }
            return;
        }
        case 13: // isect_quad_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2608ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 2624ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2640ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 2656ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 2672ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 2688ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 2704ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 2720ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r57);
                v8.z = bitcast<unsigned>(R.r61);
                v8.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 2736ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r63);
                v9.y = bitcast<unsigned>(R.r64);
                v9.z = bitcast<unsigned>(R.r65);
                v9.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 2752ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r67);
                v10.y = bitcast<unsigned>(R.r68);
                v10.z = bitcast<unsigned>(R.r69);
                v10.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 2768ull * cap)[idx] = v10;
            }
            {
                uint2 v11;
                v11.x = bitcast<unsigned>(R.r71);
                v11.y = tid;
                reinterpret_cast<uint2*>(base + 2784ull * cap)[idx] = v11;
            }
            return;
        }
        case 14: // traverse_tetrahedron
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2792ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 2808ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 2824ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 2840ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 2856ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 2872ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 2888ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 2904ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r62);
                v8.z = bitcast<unsigned>(R.r63);
                v8.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 2920ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r65);
                v9.y = bitcast<unsigned>(R.r66);
                v9.z = bitcast<unsigned>(R.r67);
                v9.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 2936ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r69);
                v10.y = bitcast<unsigned>(R.r70);
                v10.z = bitcast<unsigned>(R.r71);
                v10.w = tid;
                reinterpret_cast<uint4*>(base + 2952ull * cap)[idx] = v10;
            }
            return;
        }
        case 15: // isect_triangle_mid1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 2968ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 2984ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 3000ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 3016ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 3032ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 3048ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 3064ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r36);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 3080ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r38);
                v8.y = bitcast<unsigned>(R.r39);
                v8.z = bitcast<unsigned>(R.r40);
                v8.w = bitcast<unsigned>(R.r41);
                reinterpret_cast<uint4*>(base + 3096ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r42);
                v9.y = bitcast<unsigned>(R.r43);
                v9.z = bitcast<unsigned>(R.r44);
                v9.w = bitcast<unsigned>(R.r45);
                reinterpret_cast<uint4*>(base + 3112ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r46);
                v10.y = bitcast<unsigned>(R.r47);
                v10.z = bitcast<unsigned>(R.r48);
                v10.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 3128ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r50);
                v11.y = bitcast<unsigned>(R.r61);
                v11.z = bitcast<unsigned>(R.r62);
                v11.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 3144ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r64);
                v12.y = bitcast<unsigned>(R.r65);
                v12.z = bitcast<unsigned>(R.r66);
                v12.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 3160ull * cap)[idx] = v12;
            }
            {
                uint4 v13;
                v13.x = bitcast<unsigned>(R.r68);
                v13.y = bitcast<unsigned>(R.r69);
                v13.z = bitcast<unsigned>(R.r70);
                v13.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 3176ull * cap)[idx] = v13;
            }
            {
                unsigned v14;
                v14 = tid;
                reinterpret_cast<unsigned*>(base + 3192ull * cap)[idx] = v14;
            }
            return;
        }
        case 16: // isect_triangle_mid2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3200ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 3216ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 3232ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 3248ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 3264ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 3280ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 3296ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 3312ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r39);
                v8.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 3328ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r41);
                v9.y = bitcast<unsigned>(R.r42);
                v9.z = bitcast<unsigned>(R.r43);
                v9.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 3344ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r45);
                v10.y = bitcast<unsigned>(R.r46);
                v10.z = bitcast<unsigned>(R.r47);
                v10.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 3360ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r62);
                v11.y = bitcast<unsigned>(R.r63);
                v11.z = bitcast<unsigned>(R.r64);
                v11.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 3376ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r66);
                v12.y = bitcast<unsigned>(R.r67);
                v12.z = bitcast<unsigned>(R.r68);
                v12.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 3392ull * cap)[idx] = v12;
            }
            {
                uint4 v13;
                v13.x = bitcast<unsigned>(R.r70);
                v13.y = bitcast<unsigned>(R.r71);
                v13.z = tid;
                reinterpret_cast<uint4*>(base + 3408ull * cap)[idx] = v13;
            }
            return;
        }
        case 17: // isect_triangle_mid3
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3424ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 3440ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 3456ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 3472ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 3488ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 3504ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 3520ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 3536ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r45);
                v8.z = bitcast<unsigned>(R.r46);
                v8.w = bitcast<unsigned>(R.r47);
                reinterpret_cast<uint4*>(base + 3552ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r48);
                v9.y = bitcast<unsigned>(R.r49);
                v9.z = bitcast<unsigned>(R.r50);
                v9.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 3568ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r62);
                v10.y = bitcast<unsigned>(R.r63);
                v10.z = bitcast<unsigned>(R.r64);
                v10.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 3584ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r66);
                v11.y = bitcast<unsigned>(R.r67);
                v11.z = bitcast<unsigned>(R.r68);
                v11.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 3600ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r70);
                v12.y = bitcast<unsigned>(R.r71);
                v12.z = tid;
                reinterpret_cast<uint4*>(base + 3616ull * cap)[idx] = v12;
            }
            return;
        }
        case 18: // isect_triangle_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3632ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 3648ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 3664ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 3680ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 3696ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 3712ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 3728ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 3744ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r57);
                v8.z = bitcast<unsigned>(R.r61);
                v8.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 3760ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r63);
                v9.y = bitcast<unsigned>(R.r64);
                v9.z = bitcast<unsigned>(R.r65);
                v9.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 3776ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r67);
                v10.y = bitcast<unsigned>(R.r68);
                v10.z = bitcast<unsigned>(R.r69);
                v10.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 3792ull * cap)[idx] = v10;
            }
            {
                uint2 v11;
                v11.x = bitcast<unsigned>(R.r71);
                v11.y = tid;
                reinterpret_cast<uint2*>(base + 3808ull * cap)[idx] = v11;
            }
            return;
        }
        case 19: // traverse_sphere
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3816ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 3832ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 3848ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 3864ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 3880ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 3896ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 3912ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 3928ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r61);
                v8.y = bitcast<unsigned>(R.r62);
                v8.z = bitcast<unsigned>(R.r63);
                v8.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 3944ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r65);
                v9.y = bitcast<unsigned>(R.r66);
                v9.z = bitcast<unsigned>(R.r67);
                v9.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 3960ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r69);
                v10.y = bitcast<unsigned>(R.r70);
                v10.z = bitcast<unsigned>(R.r71);
                v10.w = tid;
                reinterpret_cast<uint4*>(base + 3976ull * cap)[idx] = v10;
            }
            return;
        }
        case 20: // traverse_solve_quadratic
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 3992ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 4008ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 4024ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 4040ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 4056ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 4072ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 4088ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r37);
                v7.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 4104ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r40);
                v8.y = bitcast<unsigned>(R.r41);
                v8.z = bitcast<unsigned>(R.r42);
                v8.w = bitcast<unsigned>(R.r43);
                reinterpret_cast<uint4*>(base + 4120ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r44);
                v9.y = bitcast<unsigned>(R.r61);
                v9.z = bitcast<unsigned>(R.r62);
                v9.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 4136ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r64);
                v10.y = bitcast<unsigned>(R.r65);
                v10.z = bitcast<unsigned>(R.r66);
                v10.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 4152ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r68);
                v11.y = bitcast<unsigned>(R.r69);
                v11.z = bitcast<unsigned>(R.r70);
                v11.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 4168ull * cap)[idx] = v11;
            }
            {
                unsigned v12;
                v12 = tid;
                reinterpret_cast<unsigned*>(base + 4184ull * cap)[idx] = v12;
            }
            return;
        }
        case 21: // sq_head1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4192ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 4208ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 4224ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 4240ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 4256ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 4272ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 4288ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r37);
                v7.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 4304ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r40);
                v8.y = bitcast<unsigned>(R.r41);
                v8.z = bitcast<unsigned>(R.r43);
                v8.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 4320ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r61);
                v9.y = bitcast<unsigned>(R.r62);
                v9.z = bitcast<unsigned>(R.r63);
                v9.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 4336ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r65);
                v10.y = bitcast<unsigned>(R.r66);
                v10.z = bitcast<unsigned>(R.r67);
                v10.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 4352ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r69);
                v11.y = bitcast<unsigned>(R.r70);
                v11.z = bitcast<unsigned>(R.r71);
                v11.w = tid;
                reinterpret_cast<uint4*>(base + 4368ull * cap)[idx] = v11;
            }
            return;
        }
        case 22: // sq_head2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4384ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 4400ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 4416ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 4432ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 4448ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 4464ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 4480ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r37);
                v7.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 4496ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r40);
                v8.y = bitcast<unsigned>(R.r41);
                v8.z = bitcast<unsigned>(R.r43);
                v8.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 4512ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r57);
                v9.y = bitcast<unsigned>(R.r62);
                v9.z = bitcast<unsigned>(R.r63);
                v9.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 4528ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r65);
                v10.y = bitcast<unsigned>(R.r66);
                v10.z = bitcast<unsigned>(R.r67);
                v10.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 4544ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r69);
                v11.y = bitcast<unsigned>(R.r70);
                v11.z = bitcast<unsigned>(R.r71);
                v11.w = tid;
                reinterpret_cast<uint4*>(base + 4560ull * cap)[idx] = v11;
            }
            return;
        }
        case 23: // sq_mid1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4576ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 4592ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 4608ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 4624ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 4640ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 4656ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 4672ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r37);
                v7.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 4688ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r40);
                v8.y = bitcast<unsigned>(R.r41);
                v8.z = bitcast<unsigned>(R.r42);
                v8.w = bitcast<unsigned>(R.r43);
                reinterpret_cast<uint4*>(base + 4704ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r44);
                v9.y = bitcast<unsigned>(R.r61);
                v9.z = bitcast<unsigned>(R.r62);
                v9.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 4720ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r64);
                v10.y = bitcast<unsigned>(R.r65);
                v10.z = bitcast<unsigned>(R.r66);
                v10.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 4736ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r68);
                v11.y = bitcast<unsigned>(R.r69);
                v11.z = bitcast<unsigned>(R.r70);
                v11.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 4752ull * cap)[idx] = v11;
            }
            {
                unsigned v12;
                v12 = tid;
                reinterpret_cast<unsigned*>(base + 4768ull * cap)[idx] = v12;
            }
            return;
        }
        case 24: // sq_mid2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4776ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 4792ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 4808ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 4824ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 4840ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 4856ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 4872ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 4888ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r39);
                v8.y = bitcast<unsigned>(R.r40);
                v8.z = bitcast<unsigned>(R.r41);
                v8.w = bitcast<unsigned>(R.r42);
                reinterpret_cast<uint4*>(base + 4904ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r43);
                v9.y = bitcast<unsigned>(R.r44);
                v9.z = bitcast<unsigned>(R.r62);
                v9.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 4920ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r64);
                v10.y = bitcast<unsigned>(R.r65);
                v10.z = bitcast<unsigned>(R.r66);
                v10.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 4936ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r68);
                v11.y = bitcast<unsigned>(R.r69);
                v11.z = bitcast<unsigned>(R.r70);
                v11.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 4952ull * cap)[idx] = v11;
            }
            {
                unsigned v12;
                v12 = tid;
                reinterpret_cast<unsigned*>(base + 4968ull * cap)[idx] = v12;
            }
            return;
        }
        case 25: // sq_mid
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 4976ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 4992ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 5008ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 5024ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 5040ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 5056ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 5072ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 5088ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r39);
                v8.y = bitcast<unsigned>(R.r40);
                v8.z = bitcast<unsigned>(R.r41);
                v8.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 5104ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r61);
                v9.y = bitcast<unsigned>(R.r62);
                v9.z = bitcast<unsigned>(R.r63);
                v9.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 5120ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r65);
                v10.y = bitcast<unsigned>(R.r66);
                v10.z = bitcast<unsigned>(R.r67);
                v10.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 5136ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r69);
                v11.y = bitcast<unsigned>(R.r70);
                v11.z = bitcast<unsigned>(R.r71);
                v11.w = tid;
                reinterpret_cast<uint4*>(base + 5152ull * cap)[idx] = v11;
            }
            return;
        }
        case 26: // sq_tail
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5168ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 5184ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 5200ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 5216ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 5232ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 5248ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 5264ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r37);
                reinterpret_cast<uint4*>(base + 5280ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r39);
                v8.y = bitcast<unsigned>(R.r40);
                v8.z = bitcast<unsigned>(R.r41);
                v8.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 5296ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r62);
                v9.y = bitcast<unsigned>(R.r63);
                v9.z = bitcast<unsigned>(R.r64);
                v9.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 5312ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r66);
                v10.y = bitcast<unsigned>(R.r67);
                v10.z = bitcast<unsigned>(R.r68);
                v10.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 5328ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r70);
                v11.y = bitcast<unsigned>(R.r71);
                v11.z = tid;
                reinterpret_cast<uint4*>(base + 5344ull * cap)[idx] = v11;
            }
            return;
        }
        case 27: // sq_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5360ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 5376ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5392ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 5408ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 5424ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 5440ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 5456ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r37);
                v7.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 5472ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r40);
                v8.y = bitcast<unsigned>(R.r41);
                v8.z = bitcast<unsigned>(R.r57);
                v8.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 5488ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r62);
                v9.y = bitcast<unsigned>(R.r63);
                v9.z = bitcast<unsigned>(R.r64);
                v9.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 5504ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r66);
                v10.y = bitcast<unsigned>(R.r67);
                v10.z = bitcast<unsigned>(R.r68);
                v10.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 5520ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r70);
                v11.y = bitcast<unsigned>(R.r71);
                v11.z = tid;
                reinterpret_cast<uint4*>(base + 5536ull * cap)[idx] = v11;
            }
            return;
        }
        case 28: // traverse_sphere_fin
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5552ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 5568ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5584ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 5600ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 5616ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 5632ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 5648ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 5664ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r57);
                v8.z = bitcast<unsigned>(R.r61);
                v8.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 5680ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r63);
                v9.y = bitcast<unsigned>(R.r64);
                v9.z = bitcast<unsigned>(R.r65);
                v9.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 5696ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r67);
                v10.y = bitcast<unsigned>(R.r68);
                v10.z = bitcast<unsigned>(R.r69);
                v10.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 5712ull * cap)[idx] = v10;
            }
            {
                uint2 v11;
                v11.x = bitcast<unsigned>(R.r71);
                v11.y = tid;
                reinterpret_cast<uint2*>(base + 5728ull * cap)[idx] = v11;
            }
            return;
        }
        case 29: // traverse_cylinder
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5736ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 5752ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5768ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 5784ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 5800ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 5816ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 5832ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 5848ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r61);
                v8.y = bitcast<unsigned>(R.r62);
                v8.z = bitcast<unsigned>(R.r63);
                v8.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 5864ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r65);
                v9.y = bitcast<unsigned>(R.r66);
                v9.z = bitcast<unsigned>(R.r67);
                v9.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 5880ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r69);
                v10.y = bitcast<unsigned>(R.r70);
                v10.z = bitcast<unsigned>(R.r71);
                v10.w = tid;
                reinterpret_cast<uint4*>(base + 5896ull * cap)[idx] = v10;
            }
            return;
        }
        case 30: // traverse_cylinder_fin
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 5912ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 5928ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 5944ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 5960ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 5976ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 5992ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 6008ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r37);
                v7.w = bitcast<unsigned>(R.r39);
                reinterpret_cast<uint4*>(base + 6024ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r40);
                v8.y = bitcast<unsigned>(R.r41);
                v8.z = bitcast<unsigned>(R.r57);
                v8.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 6040ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r62);
                v9.y = bitcast<unsigned>(R.r63);
                v9.z = bitcast<unsigned>(R.r64);
                v9.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 6056ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r66);
                v10.y = bitcast<unsigned>(R.r67);
                v10.z = bitcast<unsigned>(R.r68);
                v10.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 6072ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r70);
                v11.y = bitcast<unsigned>(R.r71);
                v11.z = tid;
                reinterpret_cast<uint4*>(base + 6088ull * cap)[idx] = v11;
            }
            return;
        }
        case 31: // traverse_disk
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 6104ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 6120ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 6136ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 6152ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 6168ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 6184ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 6200ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 6216ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r39);
                v8.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 6232ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r41);
                v9.y = bitcast<unsigned>(R.r42);
                v9.z = bitcast<unsigned>(R.r43);
                v9.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 6248ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r62);
                v10.y = bitcast<unsigned>(R.r63);
                v10.z = bitcast<unsigned>(R.r64);
                v10.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 6264ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r66);
                v11.y = bitcast<unsigned>(R.r67);
                v11.z = bitcast<unsigned>(R.r68);
                v11.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 6280ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r70);
                v12.y = bitcast<unsigned>(R.r71);
                v12.z = tid;
                reinterpret_cast<uint4*>(base + 6296ull * cap)[idx] = v12;
            }
            return;
        }
        case 32: // isect_disk_rest
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 6312ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 6328ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r14);
                reinterpret_cast<uint4*>(base + 6344ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r15);
                v3.y = bitcast<unsigned>(R.r16);
                v3.z = bitcast<unsigned>(R.r17);
                v3.w = bitcast<unsigned>(R.r18);
                reinterpret_cast<uint4*>(base + 6360ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 6376ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 6392ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 6408ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 6424ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r39);
                v8.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 6440ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r41);
                v9.y = bitcast<unsigned>(R.r61);
                v9.z = bitcast<unsigned>(R.r62);
                v9.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 6456ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r64);
                v10.y = bitcast<unsigned>(R.r65);
                v10.z = bitcast<unsigned>(R.r66);
                v10.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 6472ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r68);
                v11.y = bitcast<unsigned>(R.r69);
                v11.z = bitcast<unsigned>(R.r70);
                v11.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 6488ull * cap)[idx] = v11;
            }
            {
                unsigned v12;
                v12 = tid;
                reinterpret_cast<unsigned*>(base + 6504ull * cap)[idx] = v12;
            }
            return;
        }
        case 33: // isect_disk_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 6512ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 6528ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 6544ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 6560ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 6576ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 6592ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 6608ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 6624ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r41);
                v8.y = bitcast<unsigned>(R.r57);
                v8.z = bitcast<unsigned>(R.r61);
                v8.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 6640ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r63);
                v9.y = bitcast<unsigned>(R.r64);
                v9.z = bitcast<unsigned>(R.r65);
                v9.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 6656ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r67);
                v10.y = bitcast<unsigned>(R.r68);
                v10.z = bitcast<unsigned>(R.r69);
                v10.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 6672ull * cap)[idx] = v10;
            }
            {
                uint2 v11;
                v11.x = bitcast<unsigned>(R.r71);
                v11.y = tid;
                reinterpret_cast<uint2*>(base + 6688ull * cap)[idx] = v11;
            }
            return;
        }
        case 34: // traverse_room_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 6696ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 6712ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 6728ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r18);
                v3.w = bitcast<unsigned>(R.r19);
                reinterpret_cast<uint4*>(base + 6744ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 6760ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 6776ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 6792ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r39);
                v7.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 6808ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r61);
                v8.y = bitcast<unsigned>(R.r62);
                v8.z = bitcast<unsigned>(R.r63);
                v8.w = bitcast<unsigned>(R.r64);
                reinterpret_cast<uint4*>(base + 6824ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r65);
                v9.y = bitcast<unsigned>(R.r66);
                v9.z = bitcast<unsigned>(R.r67);
                v9.w = bitcast<unsigned>(R.r68);
                reinterpret_cast<uint4*>(base + 6840ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r69);
                v10.y = bitcast<unsigned>(R.r70);
                v10.z = bitcast<unsigned>(R.r71);
                v10.w = tid;
                reinterpret_cast<uint4*>(base + 6856ull * cap)[idx] = v10;
            }
            return;
        }
        case 35: // radiance
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 6872ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 6888ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 6904ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 6920ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 6936ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 6952ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 6968ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r35);
                v7.y = bitcast<unsigned>(R.r39);
                v7.z = bitcast<unsigned>(R.r40);
                v7.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 6984ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r62);
                v8.y = bitcast<unsigned>(R.r63);
                v8.z = bitcast<unsigned>(R.r64);
                v8.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 7000ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r66);
                v9.y = bitcast<unsigned>(R.r67);
                v9.z = bitcast<unsigned>(R.r68);
                v9.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 7016ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r70);
                v10.y = bitcast<unsigned>(R.r71);
                v10.z = tid;
                reinterpret_cast<uint4*>(base + 7032ull * cap)[idx] = v10;
            }
            return;
        }
        case 36: // set_materials
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 7048ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 7064ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 7080ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 7096ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 7112ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 7128ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r34);
                v6.y = bitcast<unsigned>(R.r35);
                v6.z = bitcast<unsigned>(R.r39);
                v6.w = bitcast<unsigned>(R.r40);
                reinterpret_cast<uint4*>(base + 7144ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r61);
                v7.y = bitcast<unsigned>(R.r69);
                v7.z = bitcast<unsigned>(R.r70);
                v7.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 7160ull * cap)[idx] = v7;
            }
            {
                unsigned v8;
                v8 = tid;
                reinterpret_cast<unsigned*>(base + 7176ull * cap)[idx] = v8;
            }
            return;
        }
        case 37: // set_polygon_normal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 7184ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 7200ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 7216ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 7232ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 7248ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 7264ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 7280ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r35);
                v7.y = bitcast<unsigned>(R.r40);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 7296ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r69);
                v8.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 7312ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r71);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 7328ull * cap)[idx] = v9;
            }
            return;
        }
        case 38: // set_disk_normal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 7336ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 7352ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 7368ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 7384ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 7400ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 7416ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 7432ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r35);
                v7.y = bitcast<unsigned>(R.r40);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 7448ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r69);
                v8.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 7464ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r71);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 7480ull * cap)[idx] = v9;
            }
            return;
        }
        case 39: // compute_sphere_normal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 7488ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 7504ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 7520ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 7536ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 7552ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 7568ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 7584ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r35);
                v7.y = bitcast<unsigned>(R.r40);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 7600ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r69);
                v8.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 7616ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r71);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 7632ull * cap)[idx] = v9;
            }
            return;
        }
        case 40: // compute_cylinder_normal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 7640ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 7656ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 7672ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 7688ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 7704ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 7720ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 7736ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r35);
                v7.y = bitcast<unsigned>(R.r40);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 7752ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r69);
                v8.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 7768ull * cap)[idx] = v8;
            }
            {
                uint2 v9;
                v9.x = bitcast<unsigned>(R.r71);
                v9.y = tid;
                reinterpret_cast<uint2*>(base + 7784ull * cap)[idx] = v9;
            }
            return;
        }
        case 41: // set_materials_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 7792ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 7808ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 7824ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 7840ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 7856ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 7872ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 7888ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r35);
                v7.y = bitcast<unsigned>(R.r40);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 7904ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r65);
                v8.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 7920ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r67);
                v9.y = bitcast<unsigned>(R.r69);
                v9.z = bitcast<unsigned>(R.r70);
                v9.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 7936ull * cap)[idx] = v9;
            }
            {
                unsigned v10;
                v10 = tid;
                reinterpret_cast<unsigned*>(base + 7952ull * cap)[idx] = v10;
            }
            return;
        }
        case 42: // test_direct
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 7960ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 7976ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 7992ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r20);
                reinterpret_cast<uint4*>(base + 8008ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 8024ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 8040ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 8056ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 8072ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r65);
                v8.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 8088ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r67);
                v9.y = bitcast<unsigned>(R.r68);
                v9.z = bitcast<unsigned>(R.r69);
                v9.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 8104ull * cap)[idx] = v9;
            }
            {
                uint2 v10;
                v10.x = bitcast<unsigned>(R.r71);
                v10.y = tid;
                reinterpret_cast<uint2*>(base + 8120ull * cap)[idx] = v10;
            }
            return;
        }
        case 43: // direct
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 8128ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 8144ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 8160ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r20);
                reinterpret_cast<uint4*>(base + 8176ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r21);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 8192ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 8208ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 8224ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 8240ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r62);
                v8.y = bitcast<unsigned>(R.r63);
                v8.z = bitcast<unsigned>(R.r64);
                v8.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 8256ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r66);
                v9.y = bitcast<unsigned>(R.r67);
                v9.z = bitcast<unsigned>(R.r68);
                v9.w = tid;
                reinterpret_cast<uint4*>(base + 8272ull * cap)[idx] = v9;
            }
            return;
        }
        case 44: // direct_pdf
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 8288ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 8304ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 8320ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 8336ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 8352ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 8368ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 8384ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r35);
                v7.y = bitcast<unsigned>(R.r40);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 8400ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r65);
                v8.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 8416ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r67);
                v9.y = bitcast<unsigned>(R.r68);
                v9.z = bitcast<unsigned>(R.r69);
                v9.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 8432ull * cap)[idx] = v9;
            }
            {
                uint2 v10;
                v10.x = bitcast<unsigned>(R.r71);
                v10.y = tid;
                reinterpret_cast<uint2*>(base + 8448ull * cap)[idx] = v10;
            }
            return;
        }
        case 45: // direct_metal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 8456ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 8472ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r9);
                v2.y = bitcast<unsigned>(R.r10);
                v2.z = bitcast<unsigned>(R.r11);
                v2.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 8488ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r13);
                v3.y = bitcast<unsigned>(R.r15);
                v3.z = bitcast<unsigned>(R.r16);
                v3.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 8504ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 8520ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 8536ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 8552ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 8568ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r62);
                v8.y = bitcast<unsigned>(R.r63);
                v8.z = bitcast<unsigned>(R.r64);
                v8.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 8584ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r66);
                v9.y = bitcast<unsigned>(R.r67);
                v9.z = bitcast<unsigned>(R.r68);
                v9.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 8600ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r70);
                v10.y = bitcast<unsigned>(R.r71);
                v10.z = tid;
                reinterpret_cast<uint4*>(base + 8616ull * cap)[idx] = v10;
            }
            return;
        }
        case 46: // window
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 8632ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 8648ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 8664ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r20);
                reinterpret_cast<uint4*>(base + 8680ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r21);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 8696ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 8712ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 8728ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 8744ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r62);
                v8.y = bitcast<unsigned>(R.r63);
                v8.z = bitcast<unsigned>(R.r64);
                v8.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 8760ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r66);
                v9.y = bitcast<unsigned>(R.r67);
                v9.z = bitcast<unsigned>(R.r68);
                v9.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 8776ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r70);
                v10.y = bitcast<unsigned>(R.r71);
                v10.z = tid;
                reinterpret_cast<uint4*>(base + 8792ull * cap)[idx] = v10;
            }
            return;
        }
        case 47: // lambert_indirect
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 8808ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r10);
                v1.z = bitcast<unsigned>(R.r11);
                v1.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 8824ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r13);
                v2.y = bitcast<unsigned>(R.r15);
                v2.z = bitcast<unsigned>(R.r16);
                v2.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 8840ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r19);
                v3.y = bitcast<unsigned>(R.r20);
                v3.z = bitcast<unsigned>(R.r21);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 8856ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 8872ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 8888ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 8904ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r61);
                v7.y = bitcast<unsigned>(R.r65);
                v7.z = bitcast<unsigned>(R.r66);
                v7.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 8920ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r68);
                v8.y = bitcast<unsigned>(R.r69);
                v8.z = bitcast<unsigned>(R.r70);
                v8.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 8936ull * cap)[idx] = v8;
            }
            {
                unsigned v9;
                v9 = tid;
                reinterpret_cast<unsigned*>(base + 8952ull * cap)[idx] = v9;
            }
            return;
        }
        case 48: // tth_begin
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 8960ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 8976ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 8992ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r20);
                reinterpret_cast<uint4*>(base + 9008ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 9024ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 9040ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r31);
                v6.z = bitcast<unsigned>(R.r32);
                v6.w = bitcast<unsigned>(R.r33);
                reinterpret_cast<uint4*>(base + 9056ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r34);
                v7.y = bitcast<unsigned>(R.r35);
                v7.z = bitcast<unsigned>(R.r61);
                v7.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 9072ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r63);
                v8.y = bitcast<unsigned>(R.r64);
                v8.z = bitcast<unsigned>(R.r65);
                v8.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 9088ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r67);
                v9.y = bitcast<unsigned>(R.r68);
                v9.z = bitcast<unsigned>(R.r69);
                v9.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 9104ull * cap)[idx] = v9;
            }
            {
                uint2 v10;
                v10.x = bitcast<unsigned>(R.r71);
                v10.y = tid;
                reinterpret_cast<uint2*>(base + 9120ull * cap)[idx] = v10;
            }
            return;
        }
        case 49: // glass
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 9128ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 9144ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 9160ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r20);
                reinterpret_cast<uint4*>(base + 9176ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r22);
                v4.y = bitcast<unsigned>(R.r23);
                v4.z = bitcast<unsigned>(R.r24);
                v4.w = bitcast<unsigned>(R.r25);
                reinterpret_cast<uint4*>(base + 9192ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r26);
                v5.y = bitcast<unsigned>(R.r27);
                v5.z = bitcast<unsigned>(R.r28);
                v5.w = bitcast<unsigned>(R.r29);
                reinterpret_cast<uint4*>(base + 9208ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r30);
                v6.y = bitcast<unsigned>(R.r34);
                v6.z = bitcast<unsigned>(R.r35);
                v6.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 9224ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r62);
                v7.y = bitcast<unsigned>(R.r63);
                v7.z = bitcast<unsigned>(R.r64);
                v7.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 9240ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r66);
                v8.y = bitcast<unsigned>(R.r67);
                v8.z = bitcast<unsigned>(R.r68);
                v8.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 9256ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r70);
                v9.y = bitcast<unsigned>(R.r71);
                v9.z = tid;
                reinterpret_cast<uint4*>(base + 9272ull * cap)[idx] = v9;
            }
            return;
        }
        case 50: // indirect_metal
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 9288ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 9304ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 9320ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r20);
                reinterpret_cast<uint4*>(base + 9336ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r21);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 9352ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 9368ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 9384ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r61);
                reinterpret_cast<uint4*>(base + 9400ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r62);
                v8.y = bitcast<unsigned>(R.r63);
                v8.z = bitcast<unsigned>(R.r64);
                v8.w = bitcast<unsigned>(R.r65);
                reinterpret_cast<uint4*>(base + 9416ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r66);
                v9.y = bitcast<unsigned>(R.r67);
                v9.z = bitcast<unsigned>(R.r68);
                v9.w = bitcast<unsigned>(R.r69);
                reinterpret_cast<uint4*>(base + 9432ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r70);
                v10.y = bitcast<unsigned>(R.r71);
                v10.z = tid;
                reinterpret_cast<uint4*>(base + 9448ull * cap)[idx] = v10;
            }
            return;
        }
        case 51: // get_slope_mid
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 9464ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 9480ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 9496ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r20);
                reinterpret_cast<uint4*>(base + 9512ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r21);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 9528ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 9544ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 9560ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 9576ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r38);
                v8.z = bitcast<unsigned>(R.r61);
                v8.w = bitcast<unsigned>(R.r62);
                reinterpret_cast<uint4*>(base + 9592ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r63);
                v9.y = bitcast<unsigned>(R.r64);
                v9.z = bitcast<unsigned>(R.r65);
                v9.w = bitcast<unsigned>(R.r66);
                reinterpret_cast<uint4*>(base + 9608ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r67);
                v10.y = bitcast<unsigned>(R.r68);
                v10.z = bitcast<unsigned>(R.r69);
                v10.w = bitcast<unsigned>(R.r70);
                reinterpret_cast<uint4*>(base + 9624ull * cap)[idx] = v10;
            }
            {
                uint2 v11;
                v11.x = bitcast<unsigned>(R.r71);
                v11.y = tid;
                reinterpret_cast<uint2*>(base + 9640ull * cap)[idx] = v11;
            }
            return;
        }
        case 52: // get_slope_end
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 9648ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r8);
                reinterpret_cast<uint4*>(base + 9664ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r10);
                v2.y = bitcast<unsigned>(R.r11);
                v2.z = bitcast<unsigned>(R.r12);
                v2.w = bitcast<unsigned>(R.r13);
                reinterpret_cast<uint4*>(base + 9680ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r14);
                v3.y = bitcast<unsigned>(R.r15);
                v3.z = bitcast<unsigned>(R.r16);
                v3.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 9696ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r19);
                v4.y = bitcast<unsigned>(R.r22);
                v4.z = bitcast<unsigned>(R.r23);
                v4.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 9712ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r25);
                v5.y = bitcast<unsigned>(R.r26);
                v5.z = bitcast<unsigned>(R.r27);
                v5.w = bitcast<unsigned>(R.r28);
                reinterpret_cast<uint4*>(base + 9728ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r29);
                v6.y = bitcast<unsigned>(R.r30);
                v6.z = bitcast<unsigned>(R.r31);
                v6.w = bitcast<unsigned>(R.r32);
                reinterpret_cast<uint4*>(base + 9744ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r33);
                v7.y = bitcast<unsigned>(R.r34);
                v7.z = bitcast<unsigned>(R.r35);
                v7.w = bitcast<unsigned>(R.r36);
                reinterpret_cast<uint4*>(base + 9760ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r37);
                v8.y = bitcast<unsigned>(R.r61);
                v8.z = bitcast<unsigned>(R.r62);
                v8.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 9776ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r64);
                v9.y = bitcast<unsigned>(R.r65);
                v9.z = bitcast<unsigned>(R.r66);
                v9.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 9792ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r68);
                v10.y = bitcast<unsigned>(R.r69);
                v10.z = bitcast<unsigned>(R.r70);
                v10.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 9808ull * cap)[idx] = v10;
            }
            {
                unsigned v11;
                v11 = tid;
                reinterpret_cast<unsigned*>(base + 9824ull * cap)[idx] = v11;
            }
            return;
        }
        case 53: // fin_sample
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 9832ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r6);
                v1.z = bitcast<unsigned>(R.r7);
                v1.w = bitcast<unsigned>(R.r10);
                reinterpret_cast<uint4*>(base + 9848ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r11);
                v2.y = bitcast<unsigned>(R.r12);
                v2.z = bitcast<unsigned>(R.r13);
                v2.w = bitcast<unsigned>(R.r15);
                reinterpret_cast<uint4*>(base + 9864ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r16);
                v3.y = bitcast<unsigned>(R.r17);
                v3.z = bitcast<unsigned>(R.r19);
                v3.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 9880ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r23);
                v4.y = bitcast<unsigned>(R.r24);
                v4.z = bitcast<unsigned>(R.r25);
                v4.w = bitcast<unsigned>(R.r26);
                reinterpret_cast<uint4*>(base + 9896ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r27);
                v5.y = bitcast<unsigned>(R.r28);
                v5.z = bitcast<unsigned>(R.r29);
                v5.w = bitcast<unsigned>(R.r30);
                reinterpret_cast<uint4*>(base + 9912ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r31);
                v6.y = bitcast<unsigned>(R.r32);
                v6.z = bitcast<unsigned>(R.r33);
                v6.w = bitcast<unsigned>(R.r34);
                reinterpret_cast<uint4*>(base + 9928ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r35);
                v7.y = bitcast<unsigned>(R.r61);
                v7.z = bitcast<unsigned>(R.r62);
                v7.w = bitcast<unsigned>(R.r63);
                reinterpret_cast<uint4*>(base + 9944ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r64);
                v8.y = bitcast<unsigned>(R.r65);
                v8.z = bitcast<unsigned>(R.r66);
                v8.w = bitcast<unsigned>(R.r67);
                reinterpret_cast<uint4*>(base + 9960ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r68);
                v9.y = bitcast<unsigned>(R.r69);
                v9.z = bitcast<unsigned>(R.r70);
                v9.w = bitcast<unsigned>(R.r71);
                reinterpret_cast<uint4*>(base + 9976ull * cap)[idx] = v9;
            }
            {
                unsigned v10;
                v10 = tid;
                reinterpret_cast<unsigned*>(base + 9992ull * cap)[idx] = v10;
            }
            return;
        }
        case 54: // fin_pixel
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r1);
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = bitcast<unsigned>(R.r3);
                v0.w = bitcast<unsigned>(R.r4);
                reinterpret_cast<uint4*>(base + 10000ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r5);
                v1.y = bitcast<unsigned>(R.r19);
                v1.z = tid;
                reinterpret_cast<uint4*>(base + 10016ull * cap)[idx] = v1;
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
            R.r14 = bitcast<unsigned int>(v0.y);
            R.r22 = bitcast<float>(v0.z);
            R.r23 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 16ull * cap)[idx];
            R.r24 = bitcast<float>(v1.x);
            R.r25 = bitcast<float>(v1.y);
            R.r26 = bitcast<float>(v1.z);
            R.r27 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 32ull * cap)[idx];
            R.r28 = bitcast<float>(v2.x);
            R.r29 = bitcast<float>(v2.y);
            R.r30 = bitcast<float>(v2.z);
            R.r31 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 48ull * cap)[idx];
            R.r32 = bitcast<float>(v3.x);
            R.r33 = bitcast<float>(v3.y);
            R.r34 = bitcast<unsigned int>(v3.z);
            R.r35 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 64ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v4.x);
            R.r62 = bitcast<float>(v4.y);
            R.r63 = bitcast<float>(v4.z);
            R.r64 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 80ull * cap)[idx];
            R.r65 = bitcast<float>(v5.x);
            R.r66 = bitcast<float>(v5.y);
            R.r67 = bitcast<float>(v5.z);
            R.r68 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 96ull * cap)[idx];
            R.r69 = bitcast<float>(v6.x);
            R.r70 = bitcast<float>(v6.y);
            R.r71 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 1: // roll
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 112ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 128ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 144ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 160ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 176ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 192ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 208ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 224ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 240ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 256ull * cap)[idx];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(base + 272ull * cap)[idx];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
        }
        case 2: // roll_split
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
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r11 = bitcast<unsigned int>(v2.z);
            R.r12 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 328ull * cap)[idx];
            R.r13 = bitcast<float>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r16 = bitcast<float>(v3.z);
            R.r17 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 344ull * cap)[idx];
            R.r18 = bitcast<unsigned int>(v4.x);
            R.r19 = bitcast<unsigned int>(v4.y);
            R.r20 = bitcast<unsigned int>(v4.z);
            R.r21 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 360ull * cap)[idx];
            R.r22 = bitcast<float>(v5.x);
            R.r23 = bitcast<float>(v5.y);
            R.r24 = bitcast<float>(v5.z);
            R.r25 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 376ull * cap)[idx];
            R.r26 = bitcast<float>(v6.x);
            R.r27 = bitcast<float>(v6.y);
            R.r28 = bitcast<float>(v6.z);
            R.r29 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 392ull * cap)[idx];
            R.r30 = bitcast<float>(v7.x);
            R.r31 = bitcast<float>(v7.y);
            R.r32 = bitcast<float>(v7.z);
            R.r33 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 408ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v8.x);
            R.r35 = bitcast<float>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 424ull * cap)[idx];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 440ull * cap)[idx];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(base + 456ull * cap)[idx];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
        }
        case 3: // sample_pixel
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 464ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 480ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r10 = bitcast<unsigned int>(v1.y);
            R.r11 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 496ull * cap)[idx];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r16 = bitcast<float>(v2.z);
            R.r17 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 512ull * cap)[idx];
            R.r18 = bitcast<unsigned int>(v3.x);
            R.r19 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<unsigned int>(v3.z);
            R.r21 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 528ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v4.x);
            R.r62 = bitcast<float>(v4.y);
            R.r63 = bitcast<float>(v4.z);
            R.r64 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 544ull * cap)[idx];
            R.r65 = bitcast<float>(v5.x);
            R.r66 = bitcast<float>(v5.y);
            R.r67 = bitcast<float>(v5.z);
            R.r68 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 560ull * cap)[idx];
            R.r69 = bitcast<float>(v6.x);
            R.r70 = bitcast<float>(v6.y);
            R.r71 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 4: // traverse_scene
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 576ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 592ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 608ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 624ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 640ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 656ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 672ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 688ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 704ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 720ull * cap)[idx];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(base + 736ull * cap)[idx];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
        }
        case 5: // traverse_box
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 776ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 792ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 808ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 824ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 840ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 856ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 872ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r61 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 888ull * cap)[idx];
            R.r64 = bitcast<float>(v9.x);
            R.r65 = bitcast<float>(v9.y);
            R.r66 = bitcast<float>(v9.z);
            R.r67 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 904ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v10.x);
            R.r69 = bitcast<float>(v10.y);
            R.r70 = bitcast<float>(v10.z);
            R.r71 = bitcast<float>(v10.w);
            const unsigned v11 = reinterpret_cast<const unsigned*>(base + 920ull * cap)[idx];
            return v11;
        }
        case 6: // isect_quad_l1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 928ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 944ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 960ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 976ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 992ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1008ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1024ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1040ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1056ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 1072ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 1088ull * cap)[idx];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r48 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 1104ull * cap)[idx];
            R.r49 = bitcast<unsigned int>(v11.x);
            R.r50 = bitcast<float>(v11.y);
            R.r58 = bitcast<float>(v11.z);
            R.r59 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 1120ull * cap)[idx];
            R.r60 = bitcast<float>(v12.x);
            R.r61 = bitcast<unsigned int>(v12.y);
            R.r62 = bitcast<float>(v12.z);
            R.r63 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(base + 1136ull * cap)[idx];
            R.r64 = bitcast<float>(v13.x);
            R.r65 = bitcast<float>(v13.y);
            R.r66 = bitcast<float>(v13.z);
            R.r67 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(base + 1152ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v14.x);
            R.r69 = bitcast<float>(v14.y);
            R.r70 = bitcast<float>(v14.z);
            R.r71 = bitcast<float>(v14.w);
            const unsigned v15 = reinterpret_cast<const unsigned*>(base + 1168ull * cap)[idx];
            return v15;
        }
        case 7: // isect_quad_l2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1176ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1192ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1208ull * cap)[idx];
            R.r10 = bitcast<unsigned int>(v2.x);
            R.r11 = bitcast<unsigned int>(v2.y);
            R.r12 = bitcast<float>(v2.z);
            R.r13 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1224ull * cap)[idx];
            R.r14 = bitcast<unsigned int>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r16 = bitcast<float>(v3.z);
            R.r17 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1240ull * cap)[idx];
            R.r18 = bitcast<unsigned int>(v4.x);
            R.r19 = bitcast<unsigned int>(v4.y);
            R.r22 = bitcast<float>(v4.z);
            R.r23 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1256ull * cap)[idx];
            R.r24 = bitcast<float>(v5.x);
            R.r25 = bitcast<float>(v5.y);
            R.r26 = bitcast<float>(v5.z);
            R.r27 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1272ull * cap)[idx];
            R.r28 = bitcast<float>(v6.x);
            R.r29 = bitcast<float>(v6.y);
            R.r30 = bitcast<float>(v6.z);
            R.r31 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1288ull * cap)[idx];
            R.r32 = bitcast<float>(v7.x);
            R.r33 = bitcast<float>(v7.y);
            R.r34 = bitcast<unsigned int>(v7.z);
            R.r35 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1304ull * cap)[idx];
            R.r36 = bitcast<float>(v8.x);
            R.r37 = bitcast<float>(v8.y);
            R.r38 = bitcast<float>(v8.z);
            R.r39 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 1320ull * cap)[idx];
            R.r40 = bitcast<unsigned int>(v9.x);
            R.r41 = bitcast<unsigned int>(v9.y);
            R.r42 = bitcast<float>(v9.z);
            R.r43 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 1336ull * cap)[idx];
            R.r44 = bitcast<unsigned int>(v10.x);
            R.r45 = bitcast<float>(v10.y);
            R.r46 = bitcast<float>(v10.z);
            R.r47 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 1352ull * cap)[idx];
            R.r48 = bitcast<unsigned int>(v11.x);
            R.r49 = bitcast<unsigned int>(v11.y);
            R.r50 = bitcast<float>(v11.z);
            R.r61 = bitcast<unsigned int>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 1368ull * cap)[idx];
            R.r62 = bitcast<float>(v12.x);
            R.r63 = bitcast<float>(v12.y);
            R.r64 = bitcast<float>(v12.z);
            R.r65 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(base + 1384ull * cap)[idx];
            R.r66 = bitcast<float>(v13.x);
            R.r67 = bitcast<float>(v13.y);
            R.r68 = bitcast<unsigned int>(v13.z);
            R.r69 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(base + 1400ull * cap)[idx];
            R.r70 = bitcast<float>(v14.x);
            R.r71 = bitcast<float>(v14.y);
            return v14.z;
        }
        case 8: // isect_quad_l3
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1416ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1432ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1448ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r11 = bitcast<unsigned int>(v2.z);
            R.r12 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1464ull * cap)[idx];
            R.r13 = bitcast<float>(v3.x);
            R.r14 = bitcast<unsigned int>(v3.y);
            R.r15 = bitcast<float>(v3.z);
            R.r16 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1480ull * cap)[idx];
            R.r17 = bitcast<float>(v4.x);
            R.r18 = bitcast<unsigned int>(v4.y);
            R.r19 = bitcast<unsigned int>(v4.z);
            R.r22 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1496ull * cap)[idx];
            R.r23 = bitcast<float>(v5.x);
            R.r24 = bitcast<float>(v5.y);
            R.r25 = bitcast<float>(v5.z);
            R.r26 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1512ull * cap)[idx];
            R.r27 = bitcast<float>(v6.x);
            R.r28 = bitcast<float>(v6.y);
            R.r29 = bitcast<float>(v6.z);
            R.r30 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1528ull * cap)[idx];
            R.r31 = bitcast<float>(v7.x);
            R.r32 = bitcast<float>(v7.y);
            R.r33 = bitcast<float>(v7.z);
            R.r34 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1544ull * cap)[idx];
            R.r35 = bitcast<float>(v8.x);
            R.r36 = bitcast<float>(v8.y);
            R.r37 = bitcast<float>(v8.z);
            R.r38 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 1560ull * cap)[idx];
            R.r39 = bitcast<float>(v9.x);
            R.r40 = bitcast<unsigned int>(v9.y);
            R.r41 = bitcast<unsigned int>(v9.z);
            R.r42 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 1576ull * cap)[idx];
            R.r43 = bitcast<unsigned int>(v10.x);
            R.r44 = bitcast<unsigned int>(v10.y);
            R.r45 = bitcast<float>(v10.z);
            R.r46 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 1592ull * cap)[idx];
            R.r47 = bitcast<float>(v11.x);
            R.r48 = bitcast<unsigned int>(v11.y);
            R.r49 = bitcast<unsigned int>(v11.z);
            R.r50 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 1608ull * cap)[idx];
            R.r62 = bitcast<float>(v12.x);
            R.r63 = bitcast<float>(v12.y);
            R.r64 = bitcast<float>(v12.z);
            R.r65 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(base + 1624ull * cap)[idx];
            R.r66 = bitcast<float>(v13.x);
            R.r67 = bitcast<float>(v13.y);
            R.r68 = bitcast<unsigned int>(v13.z);
            R.r69 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(base + 1640ull * cap)[idx];
            R.r70 = bitcast<float>(v14.x);
            R.r71 = bitcast<float>(v14.y);
            return v14.z;
        }
        case 9: // isect_quad_l4
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1656ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1672ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1688ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1704ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1720ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1736ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1752ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 1768ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 1784ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 1800ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 1816ull * cap)[idx];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r48 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 1832ull * cap)[idx];
            R.r49 = bitcast<unsigned int>(v11.x);
            R.r50 = bitcast<float>(v11.y);
            R.r62 = bitcast<float>(v11.z);
            R.r63 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 1848ull * cap)[idx];
            R.r64 = bitcast<float>(v12.x);
            R.r65 = bitcast<float>(v12.y);
            R.r66 = bitcast<float>(v12.z);
            R.r67 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(base + 1864ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v13.x);
            R.r69 = bitcast<float>(v13.y);
            R.r70 = bitcast<float>(v13.z);
            R.r71 = bitcast<float>(v13.w);
            const unsigned v14 = reinterpret_cast<const unsigned*>(base + 1880ull * cap)[idx];
            return v14;
        }
        case 10: // isect_quad_l5
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1888ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1904ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1920ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1936ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1952ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1968ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1984ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2000ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2016ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 2032ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 2048ull * cap)[idx];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r48 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 2064ull * cap)[idx];
            R.r49 = bitcast<unsigned int>(v11.x);
            R.r50 = bitcast<float>(v11.y);
            R.r51 = bitcast<float>(v11.z);
            R.r52 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 2080ull * cap)[idx];
            R.r53 = bitcast<unsigned int>(v12.x);
            R.r58 = bitcast<float>(v12.y);
            R.r59 = bitcast<float>(v12.z);
            R.r60 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(base + 2096ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v13.x);
            R.r62 = bitcast<float>(v13.y);
            R.r63 = bitcast<float>(v13.z);
            R.r64 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(base + 2112ull * cap)[idx];
            R.r65 = bitcast<float>(v14.x);
            R.r66 = bitcast<float>(v14.y);
            R.r67 = bitcast<float>(v14.z);
            R.r68 = bitcast<unsigned int>(v14.w);
            const uint4 v15 = reinterpret_cast<const uint4*>(base + 2128ull * cap)[idx];
            R.r69 = bitcast<float>(v15.x);
            R.r70 = bitcast<float>(v15.y);
            R.r71 = bitcast<float>(v15.z);
            return v15.w;
        }
        case 11: // isect_quad_l6
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2144ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2160ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2176ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2192ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2208ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2224ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2240ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2256ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2272ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 2288ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 2304ull * cap)[idx];
            R.r48 = bitcast<unsigned int>(v10.x);
            R.r49 = bitcast<unsigned int>(v10.y);
            R.r50 = bitcast<float>(v10.z);
            R.r51 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 2320ull * cap)[idx];
            R.r52 = bitcast<float>(v11.x);
            R.r53 = bitcast<unsigned int>(v11.y);
            R.r54 = bitcast<float>(v11.z);
            R.r55 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 2336ull * cap)[idx];
            R.r56 = bitcast<float>(v12.x);
            R.r61 = bitcast<unsigned int>(v12.y);
            R.r62 = bitcast<float>(v12.z);
            R.r63 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(base + 2352ull * cap)[idx];
            R.r64 = bitcast<float>(v13.x);
            R.r65 = bitcast<float>(v13.y);
            R.r66 = bitcast<float>(v13.z);
            R.r67 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(base + 2368ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v14.x);
            R.r69 = bitcast<float>(v14.y);
            R.r70 = bitcast<float>(v14.z);
            R.r71 = bitcast<float>(v14.w);
            const unsigned v15 = reinterpret_cast<const unsigned*>(base + 2384ull * cap)[idx];
            return v15;
        }
        case 12: // isect_quad_l7
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2392ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2408ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2424ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2440ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2456ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2472ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2488ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2504ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2520ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 2536ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 2552ull * cap)[idx];
            R.r48 = bitcast<unsigned int>(v10.x);
            R.r49 = bitcast<unsigned int>(v10.y);
            R.r50 = bitcast<float>(v10.z);
            R.r62 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 2568ull * cap)[idx];
            R.r63 = bitcast<float>(v11.x);
            R.r64 = bitcast<float>(v11.y);
            R.r65 = bitcast<float>(v11.z);
            R.r66 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 2584ull * cap)[idx];
            R.r67 = bitcast<float>(v12.x);
            R.r68 = bitcast<unsigned int>(v12.y);
            R.r69 = bitcast<float>(v12.z);
            R.r70 = bitcast<float>(v12.w);
            const uint2 v13 = reinterpret_cast<const uint2*>(base + 2600ull * cap)[idx];
            R.r71 = bitcast<float>(v13.x);
            return v13.y;
        }
        case 13: // isect_quad_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2608ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2624ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2640ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2656ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2672ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2688ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2704ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2720ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2736ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r57 = bitcast<unsigned int>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 2752ull * cap)[idx];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 2768ull * cap)[idx];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(base + 2784ull * cap)[idx];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
        }
        case 14: // traverse_tetrahedron
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2792ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2808ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2824ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2840ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2856ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2872ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2888ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2904ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2920ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 2936ull * cap)[idx];
            R.r65 = bitcast<float>(v9.x);
            R.r66 = bitcast<float>(v9.y);
            R.r67 = bitcast<float>(v9.z);
            R.r68 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 2952ull * cap)[idx];
            R.r69 = bitcast<float>(v10.x);
            R.r70 = bitcast<float>(v10.y);
            R.r71 = bitcast<float>(v10.z);
            return v10.w;
        }
        case 15: // isect_triangle_mid1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2968ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2984ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3000ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3016ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3032ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3048ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3064ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3080ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3096ull * cap)[idx];
            R.r38 = bitcast<float>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 3112ull * cap)[idx];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<unsigned int>(v9.y);
            R.r44 = bitcast<unsigned int>(v9.z);
            R.r45 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 3128ull * cap)[idx];
            R.r46 = bitcast<float>(v10.x);
            R.r47 = bitcast<float>(v10.y);
            R.r48 = bitcast<unsigned int>(v10.z);
            R.r49 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 3144ull * cap)[idx];
            R.r50 = bitcast<float>(v11.x);
            R.r61 = bitcast<unsigned int>(v11.y);
            R.r62 = bitcast<float>(v11.z);
            R.r63 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 3160ull * cap)[idx];
            R.r64 = bitcast<float>(v12.x);
            R.r65 = bitcast<float>(v12.y);
            R.r66 = bitcast<float>(v12.z);
            R.r67 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(base + 3176ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v13.x);
            R.r69 = bitcast<float>(v13.y);
            R.r70 = bitcast<float>(v13.z);
            R.r71 = bitcast<float>(v13.w);
            const unsigned v14 = reinterpret_cast<const unsigned*>(base + 3192ull * cap)[idx];
            return v14;
        }
        case 16: // isect_triangle_mid2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3200ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3216ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3232ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3248ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3264ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3280ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3296ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3312ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3328ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 3344ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 3360ull * cap)[idx];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r61 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 3376ull * cap)[idx];
            R.r62 = bitcast<float>(v11.x);
            R.r63 = bitcast<float>(v11.y);
            R.r64 = bitcast<float>(v11.z);
            R.r65 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 3392ull * cap)[idx];
            R.r66 = bitcast<float>(v12.x);
            R.r67 = bitcast<float>(v12.y);
            R.r68 = bitcast<unsigned int>(v12.z);
            R.r69 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(base + 3408ull * cap)[idx];
            R.r70 = bitcast<float>(v13.x);
            R.r71 = bitcast<float>(v13.y);
            return v13.z;
        }
        case 17: // isect_triangle_mid3
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3424ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3440ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3456ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3472ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3488ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3504ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3520ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3536ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3552ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r45 = bitcast<float>(v8.y);
            R.r46 = bitcast<float>(v8.z);
            R.r47 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 3568ull * cap)[idx];
            R.r48 = bitcast<unsigned int>(v9.x);
            R.r49 = bitcast<unsigned int>(v9.y);
            R.r50 = bitcast<float>(v9.z);
            R.r61 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 3584ull * cap)[idx];
            R.r62 = bitcast<float>(v10.x);
            R.r63 = bitcast<float>(v10.y);
            R.r64 = bitcast<float>(v10.z);
            R.r65 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 3600ull * cap)[idx];
            R.r66 = bitcast<float>(v11.x);
            R.r67 = bitcast<float>(v11.y);
            R.r68 = bitcast<unsigned int>(v11.z);
            R.r69 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 3616ull * cap)[idx];
            R.r70 = bitcast<float>(v12.x);
            R.r71 = bitcast<float>(v12.y);
            return v12.z;
        }
        case 18: // isect_triangle_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3632ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3648ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3664ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3680ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3696ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3712ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3728ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3744ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3760ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r57 = bitcast<unsigned int>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 3776ull * cap)[idx];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 3792ull * cap)[idx];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(base + 3808ull * cap)[idx];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
        }
        case 19: // traverse_sphere
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3816ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 3832ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 3848ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 3864ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 3880ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 3896ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 3912ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 3928ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 3944ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 3960ull * cap)[idx];
            R.r65 = bitcast<float>(v9.x);
            R.r66 = bitcast<float>(v9.y);
            R.r67 = bitcast<float>(v9.z);
            R.r68 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 3976ull * cap)[idx];
            R.r69 = bitcast<float>(v10.x);
            R.r70 = bitcast<float>(v10.y);
            R.r71 = bitcast<float>(v10.z);
            return v10.w;
        }
        case 20: // traverse_solve_quadratic
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 3992ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4008ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4024ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4040ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4056ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4072ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4088ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4104ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4120ull * cap)[idx];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r42 = bitcast<float>(v8.z);
            R.r43 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 4136ull * cap)[idx];
            R.r44 = bitcast<unsigned int>(v9.x);
            R.r61 = bitcast<unsigned int>(v9.y);
            R.r62 = bitcast<float>(v9.z);
            R.r63 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 4152ull * cap)[idx];
            R.r64 = bitcast<float>(v10.x);
            R.r65 = bitcast<float>(v10.y);
            R.r66 = bitcast<float>(v10.z);
            R.r67 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 4168ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v11.x);
            R.r69 = bitcast<float>(v11.y);
            R.r70 = bitcast<float>(v11.z);
            R.r71 = bitcast<float>(v11.w);
            const unsigned v12 = reinterpret_cast<const unsigned*>(base + 4184ull * cap)[idx];
            return v12;
        }
        case 21: // sq_head1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4192ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4208ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4224ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4240ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4256ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4272ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4288ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4304ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4320ull * cap)[idx];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r43 = bitcast<unsigned int>(v8.z);
            R.r44 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 4336ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v9.x);
            R.r62 = bitcast<float>(v9.y);
            R.r63 = bitcast<float>(v9.z);
            R.r64 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 4352ull * cap)[idx];
            R.r65 = bitcast<float>(v10.x);
            R.r66 = bitcast<float>(v10.y);
            R.r67 = bitcast<float>(v10.z);
            R.r68 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 4368ull * cap)[idx];
            R.r69 = bitcast<float>(v11.x);
            R.r70 = bitcast<float>(v11.y);
            R.r71 = bitcast<float>(v11.z);
            return v11.w;
        }
        case 22: // sq_head2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4384ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4400ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4416ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4432ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4448ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4464ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4480ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4496ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4512ull * cap)[idx];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r43 = bitcast<unsigned int>(v8.z);
            R.r44 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 4528ull * cap)[idx];
            R.r57 = bitcast<unsigned int>(v9.x);
            R.r62 = bitcast<float>(v9.y);
            R.r63 = bitcast<float>(v9.z);
            R.r64 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 4544ull * cap)[idx];
            R.r65 = bitcast<float>(v10.x);
            R.r66 = bitcast<float>(v10.y);
            R.r67 = bitcast<float>(v10.z);
            R.r68 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 4560ull * cap)[idx];
            R.r69 = bitcast<float>(v11.x);
            R.r70 = bitcast<float>(v11.y);
            R.r71 = bitcast<float>(v11.z);
            return v11.w;
        }
        case 23: // sq_mid1
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4576ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4592ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4608ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4624ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4640ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4656ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4672ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4688ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4704ull * cap)[idx];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r42 = bitcast<float>(v8.z);
            R.r43 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 4720ull * cap)[idx];
            R.r44 = bitcast<unsigned int>(v9.x);
            R.r61 = bitcast<unsigned int>(v9.y);
            R.r62 = bitcast<float>(v9.z);
            R.r63 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 4736ull * cap)[idx];
            R.r64 = bitcast<float>(v10.x);
            R.r65 = bitcast<float>(v10.y);
            R.r66 = bitcast<float>(v10.z);
            R.r67 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 4752ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v11.x);
            R.r69 = bitcast<float>(v11.y);
            R.r70 = bitcast<float>(v11.z);
            R.r71 = bitcast<float>(v11.w);
            const unsigned v12 = reinterpret_cast<const unsigned*>(base + 4768ull * cap)[idx];
            return v12;
        }
        case 24: // sq_mid2
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4776ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4792ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 4808ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 4824ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 4840ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 4856ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 4872ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 4888ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r37 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 4904ull * cap)[idx];
            R.r39 = bitcast<float>(v8.x);
            R.r40 = bitcast<unsigned int>(v8.y);
            R.r41 = bitcast<unsigned int>(v8.z);
            R.r42 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 4920ull * cap)[idx];
            R.r43 = bitcast<unsigned int>(v9.x);
            R.r44 = bitcast<unsigned int>(v9.y);
            R.r62 = bitcast<float>(v9.z);
            R.r63 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 4936ull * cap)[idx];
            R.r64 = bitcast<float>(v10.x);
            R.r65 = bitcast<float>(v10.y);
            R.r66 = bitcast<float>(v10.z);
            R.r67 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 4952ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v11.x);
            R.r69 = bitcast<float>(v11.y);
            R.r70 = bitcast<float>(v11.z);
            R.r71 = bitcast<float>(v11.w);
            const unsigned v12 = reinterpret_cast<const unsigned*>(base + 4968ull * cap)[idx];
            return v12;
        }
        case 25: // sq_mid
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 4976ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 4992ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5008ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5024ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5040ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5056ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5072ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 5088ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r37 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 5104ull * cap)[idx];
            R.r39 = bitcast<float>(v8.x);
            R.r40 = bitcast<unsigned int>(v8.y);
            R.r41 = bitcast<unsigned int>(v8.z);
            R.r44 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 5120ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v9.x);
            R.r62 = bitcast<float>(v9.y);
            R.r63 = bitcast<float>(v9.z);
            R.r64 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 5136ull * cap)[idx];
            R.r65 = bitcast<float>(v10.x);
            R.r66 = bitcast<float>(v10.y);
            R.r67 = bitcast<float>(v10.z);
            R.r68 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 5152ull * cap)[idx];
            R.r69 = bitcast<float>(v11.x);
            R.r70 = bitcast<float>(v11.y);
            R.r71 = bitcast<float>(v11.z);
            return v11.w;
        }
        case 26: // sq_tail
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5168ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5184ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5200ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5216ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5232ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5248ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5264ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 5280ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r37 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 5296ull * cap)[idx];
            R.r39 = bitcast<float>(v8.x);
            R.r40 = bitcast<unsigned int>(v8.y);
            R.r41 = bitcast<unsigned int>(v8.z);
            R.r61 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 5312ull * cap)[idx];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            R.r65 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 5328ull * cap)[idx];
            R.r66 = bitcast<float>(v10.x);
            R.r67 = bitcast<float>(v10.y);
            R.r68 = bitcast<unsigned int>(v10.z);
            R.r69 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 5344ull * cap)[idx];
            R.r70 = bitcast<float>(v11.x);
            R.r71 = bitcast<float>(v11.y);
            return v11.z;
        }
        case 27: // sq_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5360ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5376ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5392ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5408ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5424ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5440ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5456ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 5472ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 5488ull * cap)[idx];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r57 = bitcast<unsigned int>(v8.z);
            R.r61 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 5504ull * cap)[idx];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            R.r65 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 5520ull * cap)[idx];
            R.r66 = bitcast<float>(v10.x);
            R.r67 = bitcast<float>(v10.y);
            R.r68 = bitcast<unsigned int>(v10.z);
            R.r69 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 5536ull * cap)[idx];
            R.r70 = bitcast<float>(v11.x);
            R.r71 = bitcast<float>(v11.y);
            return v11.z;
        }
        case 28: // traverse_sphere_fin
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5552ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5568ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5584ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5600ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5616ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5632ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5648ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 5664ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 5680ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r57 = bitcast<unsigned int>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 5696ull * cap)[idx];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 5712ull * cap)[idx];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(base + 5728ull * cap)[idx];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
        }
        case 29: // traverse_cylinder
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5736ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5752ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5768ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5784ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5800ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5816ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 5832ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 5848ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 5864ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 5880ull * cap)[idx];
            R.r65 = bitcast<float>(v9.x);
            R.r66 = bitcast<float>(v9.y);
            R.r67 = bitcast<float>(v9.z);
            R.r68 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 5896ull * cap)[idx];
            R.r69 = bitcast<float>(v10.x);
            R.r70 = bitcast<float>(v10.y);
            R.r71 = bitcast<float>(v10.z);
            return v10.w;
        }
        case 30: // traverse_cylinder_fin
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 5912ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 5928ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 5944ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 5960ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 5976ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 5992ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 6008ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 6024ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 6040ull * cap)[idx];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r57 = bitcast<unsigned int>(v8.z);
            R.r61 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 6056ull * cap)[idx];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            R.r65 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 6072ull * cap)[idx];
            R.r66 = bitcast<float>(v10.x);
            R.r67 = bitcast<float>(v10.y);
            R.r68 = bitcast<unsigned int>(v10.z);
            R.r69 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 6088ull * cap)[idx];
            R.r70 = bitcast<float>(v11.x);
            R.r71 = bitcast<float>(v11.y);
            return v11.z;
        }
        case 31: // traverse_disk
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 6104ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 6120ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 6136ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 6152ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 6168ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 6184ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 6200ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 6216ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 6232ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 6248ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 6264ull * cap)[idx];
            R.r62 = bitcast<float>(v10.x);
            R.r63 = bitcast<float>(v10.y);
            R.r64 = bitcast<float>(v10.z);
            R.r65 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 6280ull * cap)[idx];
            R.r66 = bitcast<float>(v11.x);
            R.r67 = bitcast<float>(v11.y);
            R.r68 = bitcast<unsigned int>(v11.z);
            R.r69 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 6296ull * cap)[idx];
            R.r70 = bitcast<float>(v12.x);
            R.r71 = bitcast<float>(v12.y);
            return v12.z;
        }
        case 32: // isect_disk_rest
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 6312ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 6328ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 6344ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 6360ull * cap)[idx];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 6376ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 6392ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 6408ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 6424ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 6440ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 6456ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r61 = bitcast<unsigned int>(v9.y);
            R.r62 = bitcast<float>(v9.z);
            R.r63 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 6472ull * cap)[idx];
            R.r64 = bitcast<float>(v10.x);
            R.r65 = bitcast<float>(v10.y);
            R.r66 = bitcast<float>(v10.z);
            R.r67 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 6488ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v11.x);
            R.r69 = bitcast<float>(v11.y);
            R.r70 = bitcast<float>(v11.z);
            R.r71 = bitcast<float>(v11.w);
            const unsigned v12 = reinterpret_cast<const unsigned*>(base + 6504ull * cap)[idx];
            return v12;
        }
        case 33: // isect_disk_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 6512ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 6528ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 6544ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 6560ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 6576ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 6592ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 6608ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 6624ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 6640ull * cap)[idx];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r57 = bitcast<unsigned int>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 6656ull * cap)[idx];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 6672ull * cap)[idx];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(base + 6688ull * cap)[idx];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
        }
        case 34: // traverse_room_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 6696ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 6712ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 6728ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 6744ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r18 = bitcast<unsigned int>(v3.z);
            R.r19 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 6760ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 6776ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 6792ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 6808ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 6824ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 6840ull * cap)[idx];
            R.r65 = bitcast<float>(v9.x);
            R.r66 = bitcast<float>(v9.y);
            R.r67 = bitcast<float>(v9.z);
            R.r68 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 6856ull * cap)[idx];
            R.r69 = bitcast<float>(v10.x);
            R.r70 = bitcast<float>(v10.y);
            R.r71 = bitcast<float>(v10.z);
            return v10.w;
        }
        case 35: // radiance
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 6872ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 6888ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 6904ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 6920ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 6936ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 6952ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 6968ull * cap)[idx];
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 6984ull * cap)[idx];
            R.r35 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r40 = bitcast<unsigned int>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 7000ull * cap)[idx];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 7016ull * cap)[idx];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            R.r69 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 7032ull * cap)[idx];
            R.r70 = bitcast<float>(v10.x);
            R.r71 = bitcast<float>(v10.y);
            return v10.z;
        }
        case 36: // set_materials
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 7048ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 7064ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 7080ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 7096ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 7112ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 7128ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 7144ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v6.x);
            R.r35 = bitcast<float>(v6.y);
            R.r39 = bitcast<float>(v6.z);
            R.r40 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 7160ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v7.x);
            R.r69 = bitcast<float>(v7.y);
            R.r70 = bitcast<float>(v7.z);
            R.r71 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(base + 7176ull * cap)[idx];
            return v8;
        }
        case 37: // set_polygon_normal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 7184ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 7200ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 7216ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 7232ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 7248ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 7264ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 7280ull * cap)[idx];
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 7296ull * cap)[idx];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 7312ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r69 = bitcast<float>(v8.z);
            R.r70 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 7328ull * cap)[idx];
            R.r71 = bitcast<float>(v9.x);
            return v9.y;
        }
        case 38: // set_disk_normal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 7336ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 7352ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 7368ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 7384ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 7400ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 7416ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 7432ull * cap)[idx];
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 7448ull * cap)[idx];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 7464ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r69 = bitcast<float>(v8.z);
            R.r70 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 7480ull * cap)[idx];
            R.r71 = bitcast<float>(v9.x);
            return v9.y;
        }
        case 39: // compute_sphere_normal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 7488ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 7504ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 7520ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 7536ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 7552ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 7568ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 7584ull * cap)[idx];
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 7600ull * cap)[idx];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 7616ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r69 = bitcast<float>(v8.z);
            R.r70 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 7632ull * cap)[idx];
            R.r71 = bitcast<float>(v9.x);
            return v9.y;
        }
        case 40: // compute_cylinder_normal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 7640ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 7656ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 7672ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 7688ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 7704ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 7720ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 7736ull * cap)[idx];
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 7752ull * cap)[idx];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 7768ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r69 = bitcast<float>(v8.z);
            R.r70 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(base + 7784ull * cap)[idx];
            R.r71 = bitcast<float>(v9.x);
            return v9.y;
        }
        case 41: // set_materials_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 7792ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 7808ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 7824ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 7840ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 7856ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 7872ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 7888ull * cap)[idx];
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 7904ull * cap)[idx];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 7920ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 7936ull * cap)[idx];
            R.r67 = bitcast<float>(v9.x);
            R.r69 = bitcast<float>(v9.y);
            R.r70 = bitcast<float>(v9.z);
            R.r71 = bitcast<float>(v9.w);
            const unsigned v10 = reinterpret_cast<const unsigned*>(base + 7952ull * cap)[idx];
            return v10;
        }
        case 42: // test_direct
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 7960ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 7976ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 7992ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 8008ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 8024ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 8040ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 8056ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 8072ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 8088ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 8104ull * cap)[idx];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(base + 8120ull * cap)[idx];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
        }
        case 43: // direct
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 8128ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 8144ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 8160ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 8176ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 8192ull * cap)[idx];
            R.r21 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 8208ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 8224ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 8240ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 8256ull * cap)[idx];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 8272ull * cap)[idx];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            return v9.w;
        }
        case 44: // direct_pdf
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 8288ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 8304ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 8320ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 8336ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 8352ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 8368ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 8384ull * cap)[idx];
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 8400ull * cap)[idx];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 8416ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 8432ull * cap)[idx];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(base + 8448ull * cap)[idx];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
        }
        case 45: // direct_metal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 8456ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 8472ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 8488ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v2.x);
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r11 = bitcast<unsigned int>(v2.z);
            R.r12 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 8504ull * cap)[idx];
            R.r13 = bitcast<float>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r16 = bitcast<float>(v3.z);
            R.r17 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 8520ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 8536ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 8552ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 8568ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 8584ull * cap)[idx];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 8600ull * cap)[idx];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            R.r69 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 8616ull * cap)[idx];
            R.r70 = bitcast<float>(v10.x);
            R.r71 = bitcast<float>(v10.y);
            return v10.z;
        }
        case 46: // window
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 8632ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 8648ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 8664ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 8680ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 8696ull * cap)[idx];
            R.r21 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 8712ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 8728ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 8744ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 8760ull * cap)[idx];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 8776ull * cap)[idx];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            R.r69 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 8792ull * cap)[idx];
            R.r70 = bitcast<float>(v10.x);
            R.r71 = bitcast<float>(v10.y);
            return v10.z;
        }
        case 47: // lambert_indirect
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 8808ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 8824ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r10 = bitcast<unsigned int>(v1.y);
            R.r11 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 8840ull * cap)[idx];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r16 = bitcast<float>(v2.z);
            R.r17 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 8856ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v3.x);
            R.r20 = bitcast<unsigned int>(v3.y);
            R.r21 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 8872ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 8888ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 8904ull * cap)[idx];
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 8920ull * cap)[idx];
            R.r61 = bitcast<unsigned int>(v7.x);
            R.r65 = bitcast<float>(v7.y);
            R.r66 = bitcast<float>(v7.z);
            R.r67 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 8936ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v8.x);
            R.r69 = bitcast<float>(v8.y);
            R.r70 = bitcast<float>(v8.z);
            R.r71 = bitcast<float>(v8.w);
            const unsigned v9 = reinterpret_cast<const unsigned*>(base + 8952ull * cap)[idx];
            return v9;
        }
        case 48: // tth_begin
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 8960ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 8976ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 8992ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 9008ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 9024ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 9040ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 9056ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 9072ull * cap)[idx];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 9088ull * cap)[idx];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 9104ull * cap)[idx];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(base + 9120ull * cap)[idx];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
        }
        case 49: // glass
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 9128ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 9144ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 9160ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 9176ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 9192ull * cap)[idx];
            R.r22 = bitcast<float>(v4.x);
            R.r23 = bitcast<float>(v4.y);
            R.r24 = bitcast<float>(v4.z);
            R.r25 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 9208ull * cap)[idx];
            R.r26 = bitcast<float>(v5.x);
            R.r27 = bitcast<float>(v5.y);
            R.r28 = bitcast<float>(v5.z);
            R.r29 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 9224ull * cap)[idx];
            R.r30 = bitcast<float>(v6.x);
            R.r34 = bitcast<unsigned int>(v6.y);
            R.r35 = bitcast<float>(v6.z);
            R.r61 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 9240ull * cap)[idx];
            R.r62 = bitcast<float>(v7.x);
            R.r63 = bitcast<float>(v7.y);
            R.r64 = bitcast<float>(v7.z);
            R.r65 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 9256ull * cap)[idx];
            R.r66 = bitcast<float>(v8.x);
            R.r67 = bitcast<float>(v8.y);
            R.r68 = bitcast<unsigned int>(v8.z);
            R.r69 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 9272ull * cap)[idx];
            R.r70 = bitcast<float>(v9.x);
            R.r71 = bitcast<float>(v9.y);
            return v9.z;
        }
        case 50: // indirect_metal
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 9288ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 9304ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 9320ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 9336ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 9352ull * cap)[idx];
            R.r21 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 9368ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 9384ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 9400ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 9416ull * cap)[idx];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 9432ull * cap)[idx];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            R.r69 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 9448ull * cap)[idx];
            R.r70 = bitcast<float>(v10.x);
            R.r71 = bitcast<float>(v10.y);
            return v10.z;
        }
        case 51: // get_slope_mid
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 9464ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 9480ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 9496ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 9512ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 9528ull * cap)[idx];
            R.r21 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 9544ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 9560ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 9576ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 9592ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 9608ull * cap)[idx];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 9624ull * cap)[idx];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(base + 9640ull * cap)[idx];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
        }
        case 52: // get_slope_end
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 9648ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 9664ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r8 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 9680ull * cap)[idx];
            R.r10 = bitcast<unsigned int>(v2.x);
            R.r11 = bitcast<unsigned int>(v2.y);
            R.r12 = bitcast<float>(v2.z);
            R.r13 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 9696ull * cap)[idx];
            R.r14 = bitcast<unsigned int>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r16 = bitcast<float>(v3.z);
            R.r17 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 9712ull * cap)[idx];
            R.r19 = bitcast<unsigned int>(v4.x);
            R.r22 = bitcast<float>(v4.y);
            R.r23 = bitcast<float>(v4.z);
            R.r24 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 9728ull * cap)[idx];
            R.r25 = bitcast<float>(v5.x);
            R.r26 = bitcast<float>(v5.y);
            R.r27 = bitcast<float>(v5.z);
            R.r28 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 9744ull * cap)[idx];
            R.r29 = bitcast<float>(v6.x);
            R.r30 = bitcast<float>(v6.y);
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 9760ull * cap)[idx];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 9776ull * cap)[idx];
            R.r37 = bitcast<float>(v8.x);
            R.r61 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 9792ull * cap)[idx];
            R.r64 = bitcast<float>(v9.x);
            R.r65 = bitcast<float>(v9.y);
            R.r66 = bitcast<float>(v9.z);
            R.r67 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 9808ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v10.x);
            R.r69 = bitcast<float>(v10.y);
            R.r70 = bitcast<float>(v10.z);
            R.r71 = bitcast<float>(v10.w);
            const unsigned v11 = reinterpret_cast<const unsigned*>(base + 9824ull * cap)[idx];
            return v11;
        }
        case 53: // fin_sample
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 9832ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 9848ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 9864ull * cap)[idx];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 9880ull * cap)[idx];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r22 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 9896ull * cap)[idx];
            R.r23 = bitcast<float>(v4.x);
            R.r24 = bitcast<float>(v4.y);
            R.r25 = bitcast<float>(v4.z);
            R.r26 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 9912ull * cap)[idx];
            R.r27 = bitcast<float>(v5.x);
            R.r28 = bitcast<float>(v5.y);
            R.r29 = bitcast<float>(v5.z);
            R.r30 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 9928ull * cap)[idx];
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 9944ull * cap)[idx];
            R.r35 = bitcast<float>(v7.x);
            R.r61 = bitcast<unsigned int>(v7.y);
            R.r62 = bitcast<float>(v7.z);
            R.r63 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 9960ull * cap)[idx];
            R.r64 = bitcast<float>(v8.x);
            R.r65 = bitcast<float>(v8.y);
            R.r66 = bitcast<float>(v8.z);
            R.r67 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 9976ull * cap)[idx];
            R.r68 = bitcast<unsigned int>(v9.x);
            R.r69 = bitcast<float>(v9.y);
            R.r70 = bitcast<float>(v9.z);
            R.r71 = bitcast<float>(v9.w);
            const unsigned v10 = reinterpret_cast<const unsigned*>(base + 9992ull * cap)[idx];
            return v10;
        }
        case 54: // fin_pixel
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 10000ull * cap)[idx];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 10016ull * cap)[idx];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r19 = bitcast<unsigned int>(v1.y);
            return v1.z;
        }
        default: return 0xffffffffu;
        }
    }

    // bytes of one queue entry's slots, the largest over the queues
    static constexpr unsigned kMaxStageRow = 256u;
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
        case 0: bytes = 3584u; break;
        case 1: bytes = 5376u; break;
        case 2: bytes = 5888u; break;
        case 3: bytes = 3584u; break;
        case 4: bytes = 5376u; break;
        case 5: bytes = 5760u; break;
        case 6: bytes = 7808u; break;
        case 7: bytes = 7680u; break;
        case 8: bytes = 7680u; break;
        case 9: bytes = 7296u; break;
        case 10: bytes = 8192u; break;
        case 11: bytes = 7808u; break;
        case 12: bytes = 6912u; break;
        case 13: bytes = 5888u; break;
        case 14: bytes = 5632u; break;
        case 15: bytes = 7296u; break;
        case 16: bytes = 7168u; break;
        case 17: bytes = 6656u; break;
        case 18: bytes = 5888u; break;
        case 19: bytes = 5632u; break;
        case 20: bytes = 6272u; break;
        case 21: bytes = 6144u; break;
        case 22: bytes = 6144u; break;
        case 23: bytes = 6272u; break;
        case 24: bytes = 6272u; break;
        case 25: bytes = 6144u; break;
        case 26: bytes = 6144u; break;
        case 27: bytes = 6144u; break;
        case 28: bytes = 5888u; break;
        case 29: bytes = 5632u; break;
        case 30: bytes = 6144u; break;
        case 31: bytes = 6656u; break;
        case 32: bytes = 6272u; break;
        case 33: bytes = 5888u; break;
        case 34: bytes = 5632u; break;
        case 35: bytes = 5632u; break;
        case 36: bytes = 4224u; break;
        case 37: bytes = 4864u; break;
        case 38: bytes = 4864u; break;
        case 39: bytes = 4864u; break;
        case 40: bytes = 4864u; break;
        case 41: bytes = 5248u; break;
        case 42: bytes = 5376u; break;
        case 43: bytes = 5120u; break;
        case 44: bytes = 5376u; break;
        case 45: bytes = 5632u; break;
        case 46: bytes = 5632u; break;
        case 47: bytes = 4736u; break;
        case 48: bytes = 5376u; break;
        case 49: bytes = 5120u; break;
        case 50: bytes = 5632u; break;
        case 51: bytes = 5888u; break;
        case 52: bytes = 5760u; break;
        case 53: bytes = 5248u; break;
        case 54: bytes = 1024u; break;
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
            bulk_copy(stage + 2048u, base + 64ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 80ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 96ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 1:
            bulk_copy(stage + 0u, base + 112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 176ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 192ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 208ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 224ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 272ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 2:
            bulk_copy(stage + 0u, base + 280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 456ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 3:
            bulk_copy(stage + 0u, base + 464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 4:
            bulk_copy(stage + 0u, base + 576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 736ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 5:
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
            bulk_copy(stage + 5632u, base + 920ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 6:
            bulk_copy(stage + 0u, base + 928ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 944ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1024ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1040ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 1088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 1104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 1120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 1136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7168u, base + 1152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7680u, base + 1168ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 7:
            bulk_copy(stage + 0u, base + 1176ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1192ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1208ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1224ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1304ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1320ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 1336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 1352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 1368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 1384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7168u, base + 1400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 8:
            bulk_copy(stage + 0u, base + 1416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 1576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 1592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 1608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 1624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7168u, base + 1640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 9:
            bulk_copy(stage + 0u, base + 1656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1736ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1752ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1768ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 1784ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 1800ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 1816ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 1832ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 1848ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 1864ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7168u, base + 1880ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 10:
            bulk_copy(stage + 0u, base + 1888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1968ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 2032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 2048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 2064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 2080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 2096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7168u, base + 2112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7680u, base + 2128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 11:
            bulk_copy(stage + 0u, base + 2144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2176ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2192ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2208ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2224ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 2288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 2304ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 2320ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 2336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 2352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7168u, base + 2368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7680u, base + 2384ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 12:
            bulk_copy(stage + 0u, base + 2392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2472ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2520ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 2536ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 2552ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 2568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 2584ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 2600ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 13:
            bulk_copy(stage + 0u, base + 2608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2736ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 2752ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 2768ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 2784ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 14:
            bulk_copy(stage + 0u, base + 2792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 2936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 2952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 15:
            bulk_copy(stage + 0u, base + 2968ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 3128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 3144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 3160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 3176ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 7168u, base + 3192ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 16:
            bulk_copy(stage + 0u, base + 3200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 3360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 3376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 3392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 3408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 17:
            bulk_copy(stage + 0u, base + 3424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3472ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3520ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3536ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3552ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 3584ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 3600ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 3616ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 18:
            bulk_copy(stage + 0u, base + 3632ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3648ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3664ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3680ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 3792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 3808ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 19:
            bulk_copy(stage + 0u, base + 3816ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 3832ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 3848ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 3864ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 3880ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 3896ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 3912ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 3928ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 3944ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 3960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 3976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 20:
            bulk_copy(stage + 0u, base + 3992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4024ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4040ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 4136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 4152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 4168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 4184ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 21:
            bulk_copy(stage + 0u, base + 4192ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4208ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4224ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4304ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4320ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 4336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 4352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 4368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 22:
            bulk_copy(stage + 0u, base + 4384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 4528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 4544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 4560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 23:
            bulk_copy(stage + 0u, base + 4576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 4720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 4736ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 4752ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 4768ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 24:
            bulk_copy(stage + 0u, base + 4776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 4808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 4824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 4840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 4856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 4872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 4888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 4904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 4920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 4936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 4952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 4968ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 25:
            bulk_copy(stage + 0u, base + 4976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 4992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5024ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5040ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 5104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 5120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 5136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 5152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 26:
            bulk_copy(stage + 0u, base + 5168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 5296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 5312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 5328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 5344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 27:
            bulk_copy(stage + 0u, base + 5360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5472ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 5488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 5504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 5520ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 5536ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 28:
            bulk_copy(stage + 0u, base + 5552ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5584ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5600ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5616ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5632ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5648ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5664ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 5680ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 5696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 5712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 5728ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 29:
            bulk_copy(stage + 0u, base + 5736ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5752ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5768ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5784ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5800ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5816ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 5832ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 5848ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 5864ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 5880ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 5896ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 30:
            bulk_copy(stage + 0u, base + 5912ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 5928ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 5944ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 5960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 5976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 5992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 6008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 6024ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 6040ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 6056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 6072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 6088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 31:
            bulk_copy(stage + 0u, base + 6104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 6120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 6136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 6152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 6168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 6184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 6200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 6216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 6232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 6248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 6264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 6280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 6296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 32:
            bulk_copy(stage + 0u, base + 6312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 6328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 6344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 6360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 6376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 6392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 6408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 6424ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 6440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 6456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 6472ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 6488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 6504ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 33:
            bulk_copy(stage + 0u, base + 6512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 6528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 6544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 6560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 6576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 6592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 6608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 6624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 6640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 6656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 6672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 6688ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 34:
            bulk_copy(stage + 0u, base + 6696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 6712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 6728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 6744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 6760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 6776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 6792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 6808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 6824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 6840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 6856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 35:
            bulk_copy(stage + 0u, base + 6872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 6888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 6904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 6920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 6936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 6952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 6968ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 6984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 7000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 7016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 7032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 36:
            bulk_copy(stage + 0u, base + 7048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 7064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 7080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 7096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 7112ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 7128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 7144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 7160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 7176ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 37:
            bulk_copy(stage + 0u, base + 7184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 7200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 7216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 7232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 7248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 7264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 7280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 7296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 7312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 7328ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 38:
            bulk_copy(stage + 0u, base + 7336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 7352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 7368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 7384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 7400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 7416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 7432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 7448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 7464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 7480ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 39:
            bulk_copy(stage + 0u, base + 7488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 7504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 7520ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 7536ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 7552ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 7568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 7584ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 7600ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 7616ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 7632ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 40:
            bulk_copy(stage + 0u, base + 7640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 7656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 7672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 7688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 7704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 7720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 7736ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 7752ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 7768ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 7784ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 41:
            bulk_copy(stage + 0u, base + 7792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 7808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 7824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 7840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 7856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 7872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 7888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 7904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 7920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 7936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 7952ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 42:
            bulk_copy(stage + 0u, base + 7960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 7976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 7992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 8008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 8024ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 8040ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 8056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 8072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 8088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 8104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 8120ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 43:
            bulk_copy(stage + 0u, base + 8128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 8144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 8160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 8176ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 8192ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 8208ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 8224ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 8240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 8256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 8272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 44:
            bulk_copy(stage + 0u, base + 8288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 8304ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 8320ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 8336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 8352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 8368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 8384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 8400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 8416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 8432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 8448ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 45:
            bulk_copy(stage + 0u, base + 8456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 8472ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 8488ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 8504ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 8520ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 8536ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 8552ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 8568ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 8584ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 8600ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 8616ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 46:
            bulk_copy(stage + 0u, base + 8632ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 8648ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 8664ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 8680ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 8696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 8712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 8728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 8744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 8760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 8776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 8792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 47:
            bulk_copy(stage + 0u, base + 8808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 8824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 8840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 8856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 8872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 8888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 8904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 8920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 8936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 8952ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 48:
            bulk_copy(stage + 0u, base + 8960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 8976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 8992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 9008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 9024ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 9040ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 9056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 9072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 9088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 9104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 9120ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 49:
            bulk_copy(stage + 0u, base + 9128ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 9144ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 9160ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 9176ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 9192ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 9208ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 9224ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 9240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 9256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 9272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 50:
            bulk_copy(stage + 0u, base + 9288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 9304ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 9320ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 9336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 9352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 9368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 9384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 9400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 9416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 9432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 9448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 51:
            bulk_copy(stage + 0u, base + 9464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 9480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 9496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 9512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 9528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 9544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 9560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 9576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 9592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 9608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 9624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 9640ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 52:
            bulk_copy(stage + 0u, base + 9648ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 9664ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 9680ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 9696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 9712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 9728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 9744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 9760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 9776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 9792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 9808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 9824ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 53:
            bulk_copy(stage + 0u, base + 9832ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 9848ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 9864ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 9880ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 9896ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 9912ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 9928ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 9944ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 9960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 9976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 9992ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 54:
            bulk_copy(stage + 0u, base + 10000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 10016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
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
            R.r14 = bitcast<unsigned int>(v0.y);
            R.r22 = bitcast<float>(v0.z);
            R.r23 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r24 = bitcast<float>(v1.x);
            R.r25 = bitcast<float>(v1.y);
            R.r26 = bitcast<float>(v1.z);
            R.r27 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r28 = bitcast<float>(v2.x);
            R.r29 = bitcast<float>(v2.y);
            R.r30 = bitcast<float>(v2.z);
            R.r31 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r32 = bitcast<float>(v3.x);
            R.r33 = bitcast<float>(v3.y);
            R.r34 = bitcast<unsigned int>(v3.z);
            R.r35 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r61 = bitcast<unsigned int>(v4.x);
            R.r62 = bitcast<float>(v4.y);
            R.r63 = bitcast<float>(v4.z);
            R.r64 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r65 = bitcast<float>(v5.x);
            R.r66 = bitcast<float>(v5.y);
            R.r67 = bitcast<float>(v5.z);
            R.r68 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r69 = bitcast<float>(v6.x);
            R.r70 = bitcast<float>(v6.y);
            R.r71 = bitcast<float>(v6.z);
            return v6.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(stage + 5120u)[lane];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
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
            R.r10 = bitcast<unsigned int>(v2.y);
            R.r11 = bitcast<unsigned int>(v2.z);
            R.r12 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r13 = bitcast<float>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r16 = bitcast<float>(v3.z);
            R.r17 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r18 = bitcast<unsigned int>(v4.x);
            R.r19 = bitcast<unsigned int>(v4.y);
            R.r20 = bitcast<unsigned int>(v4.z);
            R.r21 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r22 = bitcast<float>(v5.x);
            R.r23 = bitcast<float>(v5.y);
            R.r24 = bitcast<float>(v5.z);
            R.r25 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r26 = bitcast<float>(v6.x);
            R.r27 = bitcast<float>(v6.y);
            R.r28 = bitcast<float>(v6.z);
            R.r29 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r30 = bitcast<float>(v7.x);
            R.r31 = bitcast<float>(v7.y);
            R.r32 = bitcast<float>(v7.z);
            R.r33 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r34 = bitcast<unsigned int>(v8.x);
            R.r35 = bitcast<float>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(stage + 5632u)[lane];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
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
            R.r10 = bitcast<unsigned int>(v1.y);
            R.r11 = bitcast<unsigned int>(v1.z);
            R.r12 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r13 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r16 = bitcast<float>(v2.z);
            R.r17 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r18 = bitcast<unsigned int>(v3.x);
            R.r19 = bitcast<unsigned int>(v3.y);
            R.r20 = bitcast<unsigned int>(v3.z);
            R.r21 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r61 = bitcast<unsigned int>(v4.x);
            R.r62 = bitcast<float>(v4.y);
            R.r63 = bitcast<float>(v4.z);
            R.r64 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r65 = bitcast<float>(v5.x);
            R.r66 = bitcast<float>(v5.y);
            R.r67 = bitcast<float>(v5.z);
            R.r68 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r69 = bitcast<float>(v6.x);
            R.r70 = bitcast<float>(v6.y);
            R.r71 = bitcast<float>(v6.z);
            return v6.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(stage + 5120u)[lane];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r61 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r64 = bitcast<float>(v9.x);
            R.r65 = bitcast<float>(v9.y);
            R.r66 = bitcast<float>(v9.z);
            R.r67 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r68 = bitcast<unsigned int>(v10.x);
            R.r69 = bitcast<float>(v10.y);
            R.r70 = bitcast<float>(v10.z);
            R.r71 = bitcast<float>(v10.w);
            const unsigned v11 = reinterpret_cast<const unsigned*>(stage + 5632u)[lane];
            return v11;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r48 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r49 = bitcast<unsigned int>(v11.x);
            R.r50 = bitcast<float>(v11.y);
            R.r58 = bitcast<float>(v11.z);
            R.r59 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r60 = bitcast<float>(v12.x);
            R.r61 = bitcast<unsigned int>(v12.y);
            R.r62 = bitcast<float>(v12.z);
            R.r63 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(stage + 6656u)[lane];
            R.r64 = bitcast<float>(v13.x);
            R.r65 = bitcast<float>(v13.y);
            R.r66 = bitcast<float>(v13.z);
            R.r67 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(stage + 7168u)[lane];
            R.r68 = bitcast<unsigned int>(v14.x);
            R.r69 = bitcast<float>(v14.y);
            R.r70 = bitcast<float>(v14.z);
            R.r71 = bitcast<float>(v14.w);
            const unsigned v15 = reinterpret_cast<const unsigned*>(stage + 7680u)[lane];
            return v15;
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
            R.r10 = bitcast<unsigned int>(v2.x);
            R.r11 = bitcast<unsigned int>(v2.y);
            R.r12 = bitcast<float>(v2.z);
            R.r13 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r14 = bitcast<unsigned int>(v3.x);
            R.r15 = bitcast<float>(v3.y);
            R.r16 = bitcast<float>(v3.z);
            R.r17 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r18 = bitcast<unsigned int>(v4.x);
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
            R.r31 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r32 = bitcast<float>(v7.x);
            R.r33 = bitcast<float>(v7.y);
            R.r34 = bitcast<unsigned int>(v7.z);
            R.r35 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r36 = bitcast<float>(v8.x);
            R.r37 = bitcast<float>(v8.y);
            R.r38 = bitcast<float>(v8.z);
            R.r39 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r40 = bitcast<unsigned int>(v9.x);
            R.r41 = bitcast<unsigned int>(v9.y);
            R.r42 = bitcast<float>(v9.z);
            R.r43 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r44 = bitcast<unsigned int>(v10.x);
            R.r45 = bitcast<float>(v10.y);
            R.r46 = bitcast<float>(v10.z);
            R.r47 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r48 = bitcast<unsigned int>(v11.x);
            R.r49 = bitcast<unsigned int>(v11.y);
            R.r50 = bitcast<float>(v11.z);
            R.r61 = bitcast<unsigned int>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r62 = bitcast<float>(v12.x);
            R.r63 = bitcast<float>(v12.y);
            R.r64 = bitcast<float>(v12.z);
            R.r65 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(stage + 6656u)[lane];
            R.r66 = bitcast<float>(v13.x);
            R.r67 = bitcast<float>(v13.y);
            R.r68 = bitcast<unsigned int>(v13.z);
            R.r69 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(stage + 7168u)[lane];
            R.r70 = bitcast<float>(v14.x);
            R.r71 = bitcast<float>(v14.y);
            return v14.z;
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
            R.r18 = bitcast<unsigned int>(v4.y);
            R.r19 = bitcast<unsigned int>(v4.z);
            R.r22 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r23 = bitcast<float>(v5.x);
            R.r24 = bitcast<float>(v5.y);
            R.r25 = bitcast<float>(v5.z);
            R.r26 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r27 = bitcast<float>(v6.x);
            R.r28 = bitcast<float>(v6.y);
            R.r29 = bitcast<float>(v6.z);
            R.r30 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r31 = bitcast<float>(v7.x);
            R.r32 = bitcast<float>(v7.y);
            R.r33 = bitcast<float>(v7.z);
            R.r34 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r35 = bitcast<float>(v8.x);
            R.r36 = bitcast<float>(v8.y);
            R.r37 = bitcast<float>(v8.z);
            R.r38 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r39 = bitcast<float>(v9.x);
            R.r40 = bitcast<unsigned int>(v9.y);
            R.r41 = bitcast<unsigned int>(v9.z);
            R.r42 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r43 = bitcast<unsigned int>(v10.x);
            R.r44 = bitcast<unsigned int>(v10.y);
            R.r45 = bitcast<float>(v10.z);
            R.r46 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r47 = bitcast<float>(v11.x);
            R.r48 = bitcast<unsigned int>(v11.y);
            R.r49 = bitcast<unsigned int>(v11.z);
            R.r50 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r62 = bitcast<float>(v12.x);
            R.r63 = bitcast<float>(v12.y);
            R.r64 = bitcast<float>(v12.z);
            R.r65 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(stage + 6656u)[lane];
            R.r66 = bitcast<float>(v13.x);
            R.r67 = bitcast<float>(v13.y);
            R.r68 = bitcast<unsigned int>(v13.z);
            R.r69 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(stage + 7168u)[lane];
            R.r70 = bitcast<float>(v14.x);
            R.r71 = bitcast<float>(v14.y);
            return v14.z;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r48 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r49 = bitcast<unsigned int>(v11.x);
            R.r50 = bitcast<float>(v11.y);
            R.r62 = bitcast<float>(v11.z);
            R.r63 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r64 = bitcast<float>(v12.x);
            R.r65 = bitcast<float>(v12.y);
            R.r66 = bitcast<float>(v12.z);
            R.r67 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(stage + 6656u)[lane];
            R.r68 = bitcast<unsigned int>(v13.x);
            R.r69 = bitcast<float>(v13.y);
            R.r70 = bitcast<float>(v13.z);
            R.r71 = bitcast<float>(v13.w);
            const unsigned v14 = reinterpret_cast<const unsigned*>(stage + 7168u)[lane];
            return v14;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r48 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r49 = bitcast<unsigned int>(v11.x);
            R.r50 = bitcast<float>(v11.y);
            R.r51 = bitcast<float>(v11.z);
            R.r52 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r53 = bitcast<unsigned int>(v12.x);
            R.r58 = bitcast<float>(v12.y);
            R.r59 = bitcast<float>(v12.z);
            R.r60 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(stage + 6656u)[lane];
            R.r61 = bitcast<unsigned int>(v13.x);
            R.r62 = bitcast<float>(v13.y);
            R.r63 = bitcast<float>(v13.z);
            R.r64 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(stage + 7168u)[lane];
            R.r65 = bitcast<float>(v14.x);
            R.r66 = bitcast<float>(v14.y);
            R.r67 = bitcast<float>(v14.z);
            R.r68 = bitcast<unsigned int>(v14.w);
            const uint4 v15 = reinterpret_cast<const uint4*>(stage + 7680u)[lane];
            R.r69 = bitcast<float>(v15.x);
            R.r70 = bitcast<float>(v15.y);
            R.r71 = bitcast<float>(v15.z);
            return v15.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r48 = bitcast<unsigned int>(v10.x);
            R.r49 = bitcast<unsigned int>(v10.y);
            R.r50 = bitcast<float>(v10.z);
            R.r51 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r52 = bitcast<float>(v11.x);
            R.r53 = bitcast<unsigned int>(v11.y);
            R.r54 = bitcast<float>(v11.z);
            R.r55 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r56 = bitcast<float>(v12.x);
            R.r61 = bitcast<unsigned int>(v12.y);
            R.r62 = bitcast<float>(v12.z);
            R.r63 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(stage + 6656u)[lane];
            R.r64 = bitcast<float>(v13.x);
            R.r65 = bitcast<float>(v13.y);
            R.r66 = bitcast<float>(v13.z);
            R.r67 = bitcast<float>(v13.w);
            const uint4 v14 = reinterpret_cast<const uint4*>(stage + 7168u)[lane];
            R.r68 = bitcast<unsigned int>(v14.x);
            R.r69 = bitcast<float>(v14.y);
            R.r70 = bitcast<float>(v14.z);
            R.r71 = bitcast<float>(v14.w);
            const unsigned v15 = reinterpret_cast<const unsigned*>(stage + 7680u)[lane];
            return v15;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r48 = bitcast<unsigned int>(v10.x);
            R.r49 = bitcast<unsigned int>(v10.y);
            R.r50 = bitcast<float>(v10.z);
            R.r62 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r63 = bitcast<float>(v11.x);
            R.r64 = bitcast<float>(v11.y);
            R.r65 = bitcast<float>(v11.z);
            R.r66 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r67 = bitcast<float>(v12.x);
            R.r68 = bitcast<unsigned int>(v12.y);
            R.r69 = bitcast<float>(v12.z);
            R.r70 = bitcast<float>(v12.w);
            const uint2 v13 = reinterpret_cast<const uint2*>(stage + 6656u)[lane];
            R.r71 = bitcast<float>(v13.x);
            return v13.y;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r57 = bitcast<unsigned int>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(stage + 5632u)[lane];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r65 = bitcast<float>(v9.x);
            R.r66 = bitcast<float>(v9.y);
            R.r67 = bitcast<float>(v9.z);
            R.r68 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r69 = bitcast<float>(v10.x);
            R.r70 = bitcast<float>(v10.y);
            R.r71 = bitcast<float>(v10.z);
            return v10.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r36 = bitcast<float>(v7.z);
            R.r37 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r38 = bitcast<float>(v8.x);
            R.r39 = bitcast<float>(v8.y);
            R.r40 = bitcast<unsigned int>(v8.z);
            R.r41 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r42 = bitcast<float>(v9.x);
            R.r43 = bitcast<unsigned int>(v9.y);
            R.r44 = bitcast<unsigned int>(v9.z);
            R.r45 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r46 = bitcast<float>(v10.x);
            R.r47 = bitcast<float>(v10.y);
            R.r48 = bitcast<unsigned int>(v10.z);
            R.r49 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r50 = bitcast<float>(v11.x);
            R.r61 = bitcast<unsigned int>(v11.y);
            R.r62 = bitcast<float>(v11.z);
            R.r63 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r64 = bitcast<float>(v12.x);
            R.r65 = bitcast<float>(v12.y);
            R.r66 = bitcast<float>(v12.z);
            R.r67 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(stage + 6656u)[lane];
            R.r68 = bitcast<unsigned int>(v13.x);
            R.r69 = bitcast<float>(v13.y);
            R.r70 = bitcast<float>(v13.z);
            R.r71 = bitcast<float>(v13.w);
            const unsigned v14 = reinterpret_cast<const unsigned*>(stage + 7168u)[lane];
            return v14;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r45 = bitcast<float>(v10.x);
            R.r46 = bitcast<float>(v10.y);
            R.r47 = bitcast<float>(v10.z);
            R.r61 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r62 = bitcast<float>(v11.x);
            R.r63 = bitcast<float>(v11.y);
            R.r64 = bitcast<float>(v11.z);
            R.r65 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r66 = bitcast<float>(v12.x);
            R.r67 = bitcast<float>(v12.y);
            R.r68 = bitcast<unsigned int>(v12.z);
            R.r69 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(stage + 6656u)[lane];
            R.r70 = bitcast<float>(v13.x);
            R.r71 = bitcast<float>(v13.y);
            return v13.z;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r45 = bitcast<float>(v8.y);
            R.r46 = bitcast<float>(v8.z);
            R.r47 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r48 = bitcast<unsigned int>(v9.x);
            R.r49 = bitcast<unsigned int>(v9.y);
            R.r50 = bitcast<float>(v9.z);
            R.r61 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r62 = bitcast<float>(v10.x);
            R.r63 = bitcast<float>(v10.y);
            R.r64 = bitcast<float>(v10.z);
            R.r65 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r66 = bitcast<float>(v11.x);
            R.r67 = bitcast<float>(v11.y);
            R.r68 = bitcast<unsigned int>(v11.z);
            R.r69 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r70 = bitcast<float>(v12.x);
            R.r71 = bitcast<float>(v12.y);
            return v12.z;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r57 = bitcast<unsigned int>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(stage + 5632u)[lane];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r61 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r65 = bitcast<float>(v9.x);
            R.r66 = bitcast<float>(v9.y);
            R.r67 = bitcast<float>(v9.z);
            R.r68 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r69 = bitcast<float>(v10.x);
            R.r70 = bitcast<float>(v10.y);
            R.r71 = bitcast<float>(v10.z);
            return v10.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r42 = bitcast<float>(v8.z);
            R.r43 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r44 = bitcast<unsigned int>(v9.x);
            R.r61 = bitcast<unsigned int>(v9.y);
            R.r62 = bitcast<float>(v9.z);
            R.r63 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r64 = bitcast<float>(v10.x);
            R.r65 = bitcast<float>(v10.y);
            R.r66 = bitcast<float>(v10.z);
            R.r67 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r68 = bitcast<unsigned int>(v11.x);
            R.r69 = bitcast<float>(v11.y);
            R.r70 = bitcast<float>(v11.z);
            R.r71 = bitcast<float>(v11.w);
            const unsigned v12 = reinterpret_cast<const unsigned*>(stage + 6144u)[lane];
            return v12;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r43 = bitcast<unsigned int>(v8.z);
            R.r44 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r61 = bitcast<unsigned int>(v9.x);
            R.r62 = bitcast<float>(v9.y);
            R.r63 = bitcast<float>(v9.z);
            R.r64 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r65 = bitcast<float>(v10.x);
            R.r66 = bitcast<float>(v10.y);
            R.r67 = bitcast<float>(v10.z);
            R.r68 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r69 = bitcast<float>(v11.x);
            R.r70 = bitcast<float>(v11.y);
            R.r71 = bitcast<float>(v11.z);
            return v11.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r43 = bitcast<unsigned int>(v8.z);
            R.r44 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r57 = bitcast<unsigned int>(v9.x);
            R.r62 = bitcast<float>(v9.y);
            R.r63 = bitcast<float>(v9.z);
            R.r64 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r65 = bitcast<float>(v10.x);
            R.r66 = bitcast<float>(v10.y);
            R.r67 = bitcast<float>(v10.z);
            R.r68 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r69 = bitcast<float>(v11.x);
            R.r70 = bitcast<float>(v11.y);
            R.r71 = bitcast<float>(v11.z);
            return v11.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r42 = bitcast<float>(v8.z);
            R.r43 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r44 = bitcast<unsigned int>(v9.x);
            R.r61 = bitcast<unsigned int>(v9.y);
            R.r62 = bitcast<float>(v9.z);
            R.r63 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r64 = bitcast<float>(v10.x);
            R.r65 = bitcast<float>(v10.y);
            R.r66 = bitcast<float>(v10.z);
            R.r67 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r68 = bitcast<unsigned int>(v11.x);
            R.r69 = bitcast<float>(v11.y);
            R.r70 = bitcast<float>(v11.z);
            R.r71 = bitcast<float>(v11.w);
            const unsigned v12 = reinterpret_cast<const unsigned*>(stage + 6144u)[lane];
            return v12;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r37 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r39 = bitcast<float>(v8.x);
            R.r40 = bitcast<unsigned int>(v8.y);
            R.r41 = bitcast<unsigned int>(v8.z);
            R.r42 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r43 = bitcast<unsigned int>(v9.x);
            R.r44 = bitcast<unsigned int>(v9.y);
            R.r62 = bitcast<float>(v9.z);
            R.r63 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r64 = bitcast<float>(v10.x);
            R.r65 = bitcast<float>(v10.y);
            R.r66 = bitcast<float>(v10.z);
            R.r67 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r68 = bitcast<unsigned int>(v11.x);
            R.r69 = bitcast<float>(v11.y);
            R.r70 = bitcast<float>(v11.z);
            R.r71 = bitcast<float>(v11.w);
            const unsigned v12 = reinterpret_cast<const unsigned*>(stage + 6144u)[lane];
            return v12;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r37 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r39 = bitcast<float>(v8.x);
            R.r40 = bitcast<unsigned int>(v8.y);
            R.r41 = bitcast<unsigned int>(v8.z);
            R.r44 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r61 = bitcast<unsigned int>(v9.x);
            R.r62 = bitcast<float>(v9.y);
            R.r63 = bitcast<float>(v9.z);
            R.r64 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r65 = bitcast<float>(v10.x);
            R.r66 = bitcast<float>(v10.y);
            R.r67 = bitcast<float>(v10.z);
            R.r68 = bitcast<unsigned int>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r69 = bitcast<float>(v11.x);
            R.r70 = bitcast<float>(v11.y);
            R.r71 = bitcast<float>(v11.z);
            return v11.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r37 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r39 = bitcast<float>(v8.x);
            R.r40 = bitcast<unsigned int>(v8.y);
            R.r41 = bitcast<unsigned int>(v8.z);
            R.r61 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            R.r65 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r66 = bitcast<float>(v10.x);
            R.r67 = bitcast<float>(v10.y);
            R.r68 = bitcast<unsigned int>(v10.z);
            R.r69 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r70 = bitcast<float>(v11.x);
            R.r71 = bitcast<float>(v11.y);
            return v11.z;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r57 = bitcast<unsigned int>(v8.z);
            R.r61 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            R.r65 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r66 = bitcast<float>(v10.x);
            R.r67 = bitcast<float>(v10.y);
            R.r68 = bitcast<unsigned int>(v10.z);
            R.r69 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r70 = bitcast<float>(v11.x);
            R.r71 = bitcast<float>(v11.y);
            return v11.z;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r57 = bitcast<unsigned int>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(stage + 5632u)[lane];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r61 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r65 = bitcast<float>(v9.x);
            R.r66 = bitcast<float>(v9.y);
            R.r67 = bitcast<float>(v9.z);
            R.r68 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r69 = bitcast<float>(v10.x);
            R.r70 = bitcast<float>(v10.y);
            R.r71 = bitcast<float>(v10.z);
            return v10.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r37 = bitcast<float>(v7.z);
            R.r39 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r40 = bitcast<unsigned int>(v8.x);
            R.r41 = bitcast<unsigned int>(v8.y);
            R.r57 = bitcast<unsigned int>(v8.z);
            R.r61 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r62 = bitcast<float>(v9.x);
            R.r63 = bitcast<float>(v9.y);
            R.r64 = bitcast<float>(v9.z);
            R.r65 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r66 = bitcast<float>(v10.x);
            R.r67 = bitcast<float>(v10.y);
            R.r68 = bitcast<unsigned int>(v10.z);
            R.r69 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r70 = bitcast<float>(v11.x);
            R.r71 = bitcast<float>(v11.y);
            return v11.z;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r42 = bitcast<float>(v9.y);
            R.r43 = bitcast<unsigned int>(v9.z);
            R.r44 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r62 = bitcast<float>(v10.x);
            R.r63 = bitcast<float>(v10.y);
            R.r64 = bitcast<float>(v10.z);
            R.r65 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r66 = bitcast<float>(v11.x);
            R.r67 = bitcast<float>(v11.y);
            R.r68 = bitcast<unsigned int>(v11.z);
            R.r69 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r70 = bitcast<float>(v12.x);
            R.r71 = bitcast<float>(v12.y);
            return v12.z;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r14 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r15 = bitcast<float>(v3.x);
            R.r16 = bitcast<float>(v3.y);
            R.r17 = bitcast<float>(v3.z);
            R.r18 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r39 = bitcast<float>(v8.z);
            R.r40 = bitcast<unsigned int>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r41 = bitcast<unsigned int>(v9.x);
            R.r61 = bitcast<unsigned int>(v9.y);
            R.r62 = bitcast<float>(v9.z);
            R.r63 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r64 = bitcast<float>(v10.x);
            R.r65 = bitcast<float>(v10.y);
            R.r66 = bitcast<float>(v10.z);
            R.r67 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r68 = bitcast<unsigned int>(v11.x);
            R.r69 = bitcast<float>(v11.y);
            R.r70 = bitcast<float>(v11.z);
            R.r71 = bitcast<float>(v11.w);
            const unsigned v12 = reinterpret_cast<const unsigned*>(stage + 6144u)[lane];
            return v12;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r41 = bitcast<unsigned int>(v8.x);
            R.r57 = bitcast<unsigned int>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(stage + 5632u)[lane];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r39 = bitcast<float>(v7.z);
            R.r40 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r61 = bitcast<unsigned int>(v8.x);
            R.r62 = bitcast<float>(v8.y);
            R.r63 = bitcast<float>(v8.z);
            R.r64 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r65 = bitcast<float>(v9.x);
            R.r66 = bitcast<float>(v9.y);
            R.r67 = bitcast<float>(v9.z);
            R.r68 = bitcast<unsigned int>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r69 = bitcast<float>(v10.x);
            R.r70 = bitcast<float>(v10.y);
            R.r71 = bitcast<float>(v10.z);
            return v10.w;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r35 = bitcast<float>(v7.x);
            R.r39 = bitcast<float>(v7.y);
            R.r40 = bitcast<unsigned int>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            R.r69 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r70 = bitcast<float>(v10.x);
            R.r71 = bitcast<float>(v10.y);
            return v10.z;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r34 = bitcast<unsigned int>(v6.x);
            R.r35 = bitcast<float>(v6.y);
            R.r39 = bitcast<float>(v6.z);
            R.r40 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r61 = bitcast<unsigned int>(v7.x);
            R.r69 = bitcast<float>(v7.y);
            R.r70 = bitcast<float>(v7.z);
            R.r71 = bitcast<float>(v7.w);
            const unsigned v8 = reinterpret_cast<const unsigned*>(stage + 4096u)[lane];
            return v8;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r69 = bitcast<float>(v8.z);
            R.r70 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r71 = bitcast<float>(v9.x);
            return v9.y;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r69 = bitcast<float>(v8.z);
            R.r70 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r71 = bitcast<float>(v9.x);
            return v9.y;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r69 = bitcast<float>(v8.z);
            R.r70 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r71 = bitcast<float>(v9.x);
            return v9.y;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r69 = bitcast<float>(v8.z);
            R.r70 = bitcast<float>(v8.w);
            const uint2 v9 = reinterpret_cast<const uint2*>(stage + 4608u)[lane];
            R.r71 = bitcast<float>(v9.x);
            return v9.y;
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
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r67 = bitcast<float>(v9.x);
            R.r69 = bitcast<float>(v9.y);
            R.r70 = bitcast<float>(v9.z);
            R.r71 = bitcast<float>(v9.w);
            const unsigned v10 = reinterpret_cast<const unsigned*>(stage + 5120u)[lane];
            return v10;
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(stage + 5120u)[lane];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
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
            R.r6 = bitcast<unsigned int>(v1.y);
            R.r7 = bitcast<unsigned int>(v1.z);
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r21 = bitcast<unsigned int>(v4.x);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            return v9.w;
        }
        case 44:
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r35 = bitcast<float>(v7.x);
            R.r40 = bitcast<unsigned int>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(stage + 5120u)[lane];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
        }
        case 45:
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            R.r69 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r70 = bitcast<float>(v10.x);
            R.r71 = bitcast<float>(v10.y);
            return v10.z;
        }
        case 46:
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r21 = bitcast<unsigned int>(v4.x);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            R.r69 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r70 = bitcast<float>(v10.x);
            R.r71 = bitcast<float>(v10.y);
            return v10.z;
        }
        case 47:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r1 = bitcast<unsigned int>(v0.x);
            R.r2 = bitcast<float>(v0.y);
            R.r3 = bitcast<float>(v0.z);
            R.r4 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r5 = bitcast<unsigned int>(v1.x);
            R.r10 = bitcast<unsigned int>(v1.y);
            R.r11 = bitcast<unsigned int>(v1.z);
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
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r61 = bitcast<unsigned int>(v7.x);
            R.r65 = bitcast<float>(v7.y);
            R.r66 = bitcast<float>(v7.z);
            R.r67 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r68 = bitcast<unsigned int>(v8.x);
            R.r69 = bitcast<float>(v8.y);
            R.r70 = bitcast<float>(v8.z);
            R.r71 = bitcast<float>(v8.w);
            const unsigned v9 = reinterpret_cast<const unsigned*>(stage + 4608u)[lane];
            return v9;
        }
        case 48:
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
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
            R.r31 = bitcast<float>(v6.y);
            R.r32 = bitcast<float>(v6.z);
            R.r33 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r34 = bitcast<unsigned int>(v7.x);
            R.r35 = bitcast<float>(v7.y);
            R.r61 = bitcast<unsigned int>(v7.z);
            R.r62 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r63 = bitcast<float>(v8.x);
            R.r64 = bitcast<float>(v8.y);
            R.r65 = bitcast<float>(v8.z);
            R.r66 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r67 = bitcast<float>(v9.x);
            R.r68 = bitcast<unsigned int>(v9.y);
            R.r69 = bitcast<float>(v9.z);
            R.r70 = bitcast<float>(v9.w);
            const uint2 v10 = reinterpret_cast<const uint2*>(stage + 5120u)[lane];
            R.r71 = bitcast<float>(v10.x);
            return v10.y;
        }
        case 49:
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
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
            R.r34 = bitcast<unsigned int>(v6.y);
            R.r35 = bitcast<float>(v6.z);
            R.r61 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r62 = bitcast<float>(v7.x);
            R.r63 = bitcast<float>(v7.y);
            R.r64 = bitcast<float>(v7.z);
            R.r65 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r66 = bitcast<float>(v8.x);
            R.r67 = bitcast<float>(v8.y);
            R.r68 = bitcast<unsigned int>(v8.z);
            R.r69 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r70 = bitcast<float>(v9.x);
            R.r71 = bitcast<float>(v9.y);
            return v9.z;
        }
        case 50:
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r21 = bitcast<unsigned int>(v4.x);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r61 = bitcast<unsigned int>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r62 = bitcast<float>(v8.x);
            R.r63 = bitcast<float>(v8.y);
            R.r64 = bitcast<float>(v8.z);
            R.r65 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r66 = bitcast<float>(v9.x);
            R.r67 = bitcast<float>(v9.y);
            R.r68 = bitcast<unsigned int>(v9.z);
            R.r69 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r70 = bitcast<float>(v10.x);
            R.r71 = bitcast<float>(v10.y);
            return v10.z;
        }
        case 51:
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
            R.r12 = bitcast<float>(v2.y);
            R.r13 = bitcast<float>(v2.z);
            R.r15 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r16 = bitcast<float>(v3.x);
            R.r17 = bitcast<float>(v3.y);
            R.r19 = bitcast<unsigned int>(v3.z);
            R.r20 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r21 = bitcast<unsigned int>(v4.x);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r38 = bitcast<float>(v8.y);
            R.r61 = bitcast<unsigned int>(v8.z);
            R.r62 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r63 = bitcast<float>(v9.x);
            R.r64 = bitcast<float>(v9.y);
            R.r65 = bitcast<float>(v9.z);
            R.r66 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r67 = bitcast<float>(v10.x);
            R.r68 = bitcast<unsigned int>(v10.y);
            R.r69 = bitcast<float>(v10.z);
            R.r70 = bitcast<float>(v10.w);
            const uint2 v11 = reinterpret_cast<const uint2*>(stage + 5632u)[lane];
            R.r71 = bitcast<float>(v11.x);
            return v11.y;
        }
        case 52:
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
            R.r10 = bitcast<unsigned int>(v2.x);
            R.r11 = bitcast<unsigned int>(v2.y);
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
            R.r31 = bitcast<float>(v6.z);
            R.r32 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r33 = bitcast<float>(v7.x);
            R.r34 = bitcast<unsigned int>(v7.y);
            R.r35 = bitcast<float>(v7.z);
            R.r36 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r37 = bitcast<float>(v8.x);
            R.r61 = bitcast<unsigned int>(v8.y);
            R.r62 = bitcast<float>(v8.z);
            R.r63 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r64 = bitcast<float>(v9.x);
            R.r65 = bitcast<float>(v9.y);
            R.r66 = bitcast<float>(v9.z);
            R.r67 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r68 = bitcast<unsigned int>(v10.x);
            R.r69 = bitcast<float>(v10.y);
            R.r70 = bitcast<float>(v10.z);
            R.r71 = bitcast<float>(v10.w);
            const unsigned v11 = reinterpret_cast<const unsigned*>(stage + 5632u)[lane];
            return v11;
        }
        case 53:
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
            R.r10 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r11 = bitcast<unsigned int>(v2.x);
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
            R.r31 = bitcast<float>(v6.x);
            R.r32 = bitcast<float>(v6.y);
            R.r33 = bitcast<float>(v6.z);
            R.r34 = bitcast<unsigned int>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r35 = bitcast<float>(v7.x);
            R.r61 = bitcast<unsigned int>(v7.y);
            R.r62 = bitcast<float>(v7.z);
            R.r63 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r64 = bitcast<float>(v8.x);
            R.r65 = bitcast<float>(v8.y);
            R.r66 = bitcast<float>(v8.z);
            R.r67 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r68 = bitcast<unsigned int>(v9.x);
            R.r69 = bitcast<float>(v9.y);
            R.r70 = bitcast<float>(v9.z);
            R.r71 = bitcast<float>(v9.w);
            const unsigned v10 = reinterpret_cast<const unsigned*>(stage + 5120u)[lane];
            return v10;
        }
        case 54:
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
const uint32_t kInstrs[] = {29, 297, 2, 37, 10, 31, 11, 20, 3, 19, 10, 13, 22, 7, 28, 12, 15, 7, 7, 25, 3, 3, 3, 5, 11, 4, 3, 2, 4, 13, 15, 14, 16, 13, 5, 14, 31, 4, 19, 12, 12, 8, 4, 42, 36, 113, 42, 69, 37, 82, 27, 53, 128, 23, 5};
const uint32_t kLive[] = {108, 164, 180, 108, 164, 176, 240, 232, 232, 224, 252, 240, 212, 180, 172, 224, 216, 200, 180, 172, 192, 188, 188, 192, 192, 188, 184, 184, 180, 172, 184, 200, 192, 180, 172, 168, 128, 148, 148, 148, 148, 160, 164, 156, 164, 168, 168, 144, 164, 152, 168, 180, 176, 160, 24};

const loom_b200_kernel_info kInfo = {
    "pt2_const_512", "89a954cc5f4ea54a", 1u, 5u, kInTypes, kOutTypes, kInNames, kOutNames,
    55u, 72u, 288u, 71u, kInstrs, kLive};

const uint32_t kQRegs0[] = {1u, 14u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes0[] = {LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames0[] = {"ppp", "tmp0", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs0[] = {0ull, 0ull, 0ull, 0ull, 16ull, 16ull, 16ull, 16ull, 32ull, 32ull, 32ull, 32ull, 48ull, 48ull, 48ull, 48ull, 64ull, 64ull, 64ull, 64ull, 80ull, 80ull, 80ull, 80ull, 96ull, 96ull, 96ull};
const unsigned kQSubs0[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths0[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs1[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes1[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames1[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs1[] = {112ull, 112ull, 112ull, 112ull, 128ull, 128ull, 128ull, 128ull, 144ull, 144ull, 144ull, 144ull, 160ull, 160ull, 160ull, 160ull, 176ull, 176ull, 176ull, 176ull, 192ull, 192ull, 192ull, 192ull, 208ull, 208ull, 208ull, 208ull, 224ull, 224ull, 224ull, 224ull, 240ull, 240ull, 240ull, 240ull, 256ull, 256ull, 256ull, 256ull, 272ull};
const unsigned kQSubs1[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths1[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs2[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 20u, 21u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes2[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames2[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "tmp1", "tmp2", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "u0", "u1", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs2[] = {280ull, 280ull, 280ull, 280ull, 296ull, 296ull, 296ull, 296ull, 312ull, 312ull, 312ull, 312ull, 328ull, 328ull, 328ull, 328ull, 344ull, 344ull, 344ull, 344ull, 360ull, 360ull, 360ull, 360ull, 376ull, 376ull, 376ull, 376ull, 392ull, 392ull, 392ull, 392ull, 408ull, 408ull, 408ull, 408ull, 424ull, 424ull, 424ull, 424ull, 440ull, 440ull, 440ull, 440ull, 456ull};
const unsigned kQSubs2[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths2[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs3[] = {1u, 2u, 3u, 4u, 5u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 20u, 21u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes3[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames3[] = {"ppp", "L0", "L1", "L2", "rc", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "u0", "u1", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs3[] = {464ull, 464ull, 464ull, 464ull, 480ull, 480ull, 480ull, 480ull, 496ull, 496ull, 496ull, 496ull, 512ull, 512ull, 512ull, 512ull, 528ull, 528ull, 528ull, 528ull, 544ull, 544ull, 544ull, 544ull, 560ull, 560ull, 560ull};
const unsigned kQSubs3[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths3[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs4[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes4[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames4[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs4[] = {576ull, 576ull, 576ull, 576ull, 592ull, 592ull, 592ull, 592ull, 608ull, 608ull, 608ull, 608ull, 624ull, 624ull, 624ull, 624ull, 640ull, 640ull, 640ull, 640ull, 656ull, 656ull, 656ull, 656ull, 672ull, 672ull, 672ull, 672ull, 688ull, 688ull, 688ull, 688ull, 704ull, 704ull, 704ull, 704ull, 720ull, 720ull, 720ull, 720ull, 736ull};
const unsigned kQSubs4[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths4[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs5[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 41u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes5[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames5[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs5[] = {744ull, 744ull, 744ull, 744ull, 760ull, 760ull, 760ull, 760ull, 776ull, 776ull, 776ull, 776ull, 792ull, 792ull, 792ull, 792ull, 808ull, 808ull, 808ull, 808ull, 824ull, 824ull, 824ull, 824ull, 840ull, 840ull, 840ull, 840ull, 856ull, 856ull, 856ull, 856ull, 872ull, 872ull, 872ull, 872ull, 888ull, 888ull, 888ull, 888ull, 904ull, 904ull, 904ull, 904ull};
const unsigned kQSubs5[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths5[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs6[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 48u, 49u, 50u, 58u, 59u, 60u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes6[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames6[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "vr60", "vr61", "vr62", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs6[] = {928ull, 928ull, 928ull, 928ull, 944ull, 944ull, 944ull, 944ull, 960ull, 960ull, 960ull, 960ull, 976ull, 976ull, 976ull, 976ull, 992ull, 992ull, 992ull, 992ull, 1008ull, 1008ull, 1008ull, 1008ull, 1024ull, 1024ull, 1024ull, 1024ull, 1040ull, 1040ull, 1040ull, 1040ull, 1056ull, 1056ull, 1056ull, 1056ull, 1072ull, 1072ull, 1072ull, 1072ull, 1088ull, 1088ull, 1088ull, 1088ull, 1104ull, 1104ull, 1104ull, 1104ull, 1120ull, 1120ull, 1120ull, 1120ull, 1136ull, 1136ull, 1136ull, 1136ull, 1152ull, 1152ull, 1152ull, 1152ull};
const unsigned kQSubs6[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths6[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs7[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 48u, 49u, 50u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes7[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames7[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "tmp1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs7[] = {1176ull, 1176ull, 1176ull, 1176ull, 1192ull, 1192ull, 1192ull, 1192ull, 1208ull, 1208ull, 1208ull, 1208ull, 1224ull, 1224ull, 1224ull, 1224ull, 1240ull, 1240ull, 1240ull, 1240ull, 1256ull, 1256ull, 1256ull, 1256ull, 1272ull, 1272ull, 1272ull, 1272ull, 1288ull, 1288ull, 1288ull, 1288ull, 1304ull, 1304ull, 1304ull, 1304ull, 1320ull, 1320ull, 1320ull, 1320ull, 1336ull, 1336ull, 1336ull, 1336ull, 1352ull, 1352ull, 1352ull, 1352ull, 1368ull, 1368ull, 1368ull, 1368ull, 1384ull, 1384ull, 1384ull, 1384ull, 1400ull, 1400ull};
const unsigned kQSubs7[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths7[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs8[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 48u, 49u, 50u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes8[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames8[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "tmp1", "tmp2", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs8[] = {1416ull, 1416ull, 1416ull, 1416ull, 1432ull, 1432ull, 1432ull, 1432ull, 1448ull, 1448ull, 1448ull, 1448ull, 1464ull, 1464ull, 1464ull, 1464ull, 1480ull, 1480ull, 1480ull, 1480ull, 1496ull, 1496ull, 1496ull, 1496ull, 1512ull, 1512ull, 1512ull, 1512ull, 1528ull, 1528ull, 1528ull, 1528ull, 1544ull, 1544ull, 1544ull, 1544ull, 1560ull, 1560ull, 1560ull, 1560ull, 1576ull, 1576ull, 1576ull, 1576ull, 1592ull, 1592ull, 1592ull, 1592ull, 1608ull, 1608ull, 1608ull, 1608ull, 1624ull, 1624ull, 1624ull, 1624ull, 1640ull, 1640ull};
const unsigned kQSubs8[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths8[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs9[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 48u, 49u, 50u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes9[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames9[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs9[] = {1656ull, 1656ull, 1656ull, 1656ull, 1672ull, 1672ull, 1672ull, 1672ull, 1688ull, 1688ull, 1688ull, 1688ull, 1704ull, 1704ull, 1704ull, 1704ull, 1720ull, 1720ull, 1720ull, 1720ull, 1736ull, 1736ull, 1736ull, 1736ull, 1752ull, 1752ull, 1752ull, 1752ull, 1768ull, 1768ull, 1768ull, 1768ull, 1784ull, 1784ull, 1784ull, 1784ull, 1800ull, 1800ull, 1800ull, 1800ull, 1816ull, 1816ull, 1816ull, 1816ull, 1832ull, 1832ull, 1832ull, 1832ull, 1848ull, 1848ull, 1848ull, 1848ull, 1864ull, 1864ull, 1864ull, 1864ull};
const unsigned kQSubs9[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths9[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs10[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 53u, 58u, 59u, 60u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes10[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames10[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "vr40", "vr41", "vr42", "vr60", "vr61", "vr62", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs10[] = {1888ull, 1888ull, 1888ull, 1888ull, 1904ull, 1904ull, 1904ull, 1904ull, 1920ull, 1920ull, 1920ull, 1920ull, 1936ull, 1936ull, 1936ull, 1936ull, 1952ull, 1952ull, 1952ull, 1952ull, 1968ull, 1968ull, 1968ull, 1968ull, 1984ull, 1984ull, 1984ull, 1984ull, 2000ull, 2000ull, 2000ull, 2000ull, 2016ull, 2016ull, 2016ull, 2016ull, 2032ull, 2032ull, 2032ull, 2032ull, 2048ull, 2048ull, 2048ull, 2048ull, 2064ull, 2064ull, 2064ull, 2064ull, 2080ull, 2080ull, 2080ull, 2080ull, 2096ull, 2096ull, 2096ull, 2096ull, 2112ull, 2112ull, 2112ull, 2112ull, 2128ull, 2128ull, 2128ull};
const unsigned kQSubs10[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths10[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs11[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 48u, 49u, 50u, 51u, 52u, 53u, 54u, 55u, 56u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes11[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames11[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr30", "vr31", "vr32", "vr40", "vr41", "vr42", "vr50", "vr51", "vr52", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs11[] = {2144ull, 2144ull, 2144ull, 2144ull, 2160ull, 2160ull, 2160ull, 2160ull, 2176ull, 2176ull, 2176ull, 2176ull, 2192ull, 2192ull, 2192ull, 2192ull, 2208ull, 2208ull, 2208ull, 2208ull, 2224ull, 2224ull, 2224ull, 2224ull, 2240ull, 2240ull, 2240ull, 2240ull, 2256ull, 2256ull, 2256ull, 2256ull, 2272ull, 2272ull, 2272ull, 2272ull, 2288ull, 2288ull, 2288ull, 2288ull, 2304ull, 2304ull, 2304ull, 2304ull, 2320ull, 2320ull, 2320ull, 2320ull, 2336ull, 2336ull, 2336ull, 2336ull, 2352ull, 2352ull, 2352ull, 2352ull, 2368ull, 2368ull, 2368ull, 2368ull};
const unsigned kQSubs11[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths11[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs12[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 48u, 49u, 50u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes12[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames12[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr30", "vr31", "vr32", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs12[] = {2392ull, 2392ull, 2392ull, 2392ull, 2408ull, 2408ull, 2408ull, 2408ull, 2424ull, 2424ull, 2424ull, 2424ull, 2440ull, 2440ull, 2440ull, 2440ull, 2456ull, 2456ull, 2456ull, 2456ull, 2472ull, 2472ull, 2472ull, 2472ull, 2488ull, 2488ull, 2488ull, 2488ull, 2504ull, 2504ull, 2504ull, 2504ull, 2520ull, 2520ull, 2520ull, 2520ull, 2536ull, 2536ull, 2536ull, 2536ull, 2552ull, 2552ull, 2552ull, 2552ull, 2568ull, 2568ull, 2568ull, 2568ull, 2584ull, 2584ull, 2584ull, 2584ull, 2600ull};
const unsigned kQSubs12[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths12[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs13[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 41u, 57u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes13[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames13[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "hit", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs13[] = {2608ull, 2608ull, 2608ull, 2608ull, 2624ull, 2624ull, 2624ull, 2624ull, 2640ull, 2640ull, 2640ull, 2640ull, 2656ull, 2656ull, 2656ull, 2656ull, 2672ull, 2672ull, 2672ull, 2672ull, 2688ull, 2688ull, 2688ull, 2688ull, 2704ull, 2704ull, 2704ull, 2704ull, 2720ull, 2720ull, 2720ull, 2720ull, 2736ull, 2736ull, 2736ull, 2736ull, 2752ull, 2752ull, 2752ull, 2752ull, 2768ull, 2768ull, 2768ull, 2768ull, 2784ull};
const unsigned kQSubs13[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths13[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs14[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 41u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes14[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames14[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs14[] = {2792ull, 2792ull, 2792ull, 2792ull, 2808ull, 2808ull, 2808ull, 2808ull, 2824ull, 2824ull, 2824ull, 2824ull, 2840ull, 2840ull, 2840ull, 2840ull, 2856ull, 2856ull, 2856ull, 2856ull, 2872ull, 2872ull, 2872ull, 2872ull, 2888ull, 2888ull, 2888ull, 2888ull, 2904ull, 2904ull, 2904ull, 2904ull, 2920ull, 2920ull, 2920ull, 2920ull, 2936ull, 2936ull, 2936ull, 2936ull, 2952ull, 2952ull, 2952ull};
const unsigned kQSubs14[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths14[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs15[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 48u, 49u, 50u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes15[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames15[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs15[] = {2968ull, 2968ull, 2968ull, 2968ull, 2984ull, 2984ull, 2984ull, 2984ull, 3000ull, 3000ull, 3000ull, 3000ull, 3016ull, 3016ull, 3016ull, 3016ull, 3032ull, 3032ull, 3032ull, 3032ull, 3048ull, 3048ull, 3048ull, 3048ull, 3064ull, 3064ull, 3064ull, 3064ull, 3080ull, 3080ull, 3080ull, 3080ull, 3096ull, 3096ull, 3096ull, 3096ull, 3112ull, 3112ull, 3112ull, 3112ull, 3128ull, 3128ull, 3128ull, 3128ull, 3144ull, 3144ull, 3144ull, 3144ull, 3160ull, 3160ull, 3160ull, 3160ull, 3176ull, 3176ull, 3176ull, 3176ull};
const unsigned kQSubs15[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths15[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs16[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes16[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames16[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs16[] = {3200ull, 3200ull, 3200ull, 3200ull, 3216ull, 3216ull, 3216ull, 3216ull, 3232ull, 3232ull, 3232ull, 3232ull, 3248ull, 3248ull, 3248ull, 3248ull, 3264ull, 3264ull, 3264ull, 3264ull, 3280ull, 3280ull, 3280ull, 3280ull, 3296ull, 3296ull, 3296ull, 3296ull, 3312ull, 3312ull, 3312ull, 3312ull, 3328ull, 3328ull, 3328ull, 3328ull, 3344ull, 3344ull, 3344ull, 3344ull, 3360ull, 3360ull, 3360ull, 3360ull, 3376ull, 3376ull, 3376ull, 3376ull, 3392ull, 3392ull, 3392ull, 3392ull, 3408ull, 3408ull};
const unsigned kQSubs16[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths16[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs17[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 41u, 45u, 46u, 47u, 48u, 49u, 50u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes17[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames17[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs17[] = {3424ull, 3424ull, 3424ull, 3424ull, 3440ull, 3440ull, 3440ull, 3440ull, 3456ull, 3456ull, 3456ull, 3456ull, 3472ull, 3472ull, 3472ull, 3472ull, 3488ull, 3488ull, 3488ull, 3488ull, 3504ull, 3504ull, 3504ull, 3504ull, 3520ull, 3520ull, 3520ull, 3520ull, 3536ull, 3536ull, 3536ull, 3536ull, 3552ull, 3552ull, 3552ull, 3552ull, 3568ull, 3568ull, 3568ull, 3568ull, 3584ull, 3584ull, 3584ull, 3584ull, 3600ull, 3600ull, 3600ull, 3600ull, 3616ull, 3616ull};
const unsigned kQSubs17[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths17[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs18[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 41u, 57u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes18[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames18[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "hit", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs18[] = {3632ull, 3632ull, 3632ull, 3632ull, 3648ull, 3648ull, 3648ull, 3648ull, 3664ull, 3664ull, 3664ull, 3664ull, 3680ull, 3680ull, 3680ull, 3680ull, 3696ull, 3696ull, 3696ull, 3696ull, 3712ull, 3712ull, 3712ull, 3712ull, 3728ull, 3728ull, 3728ull, 3728ull, 3744ull, 3744ull, 3744ull, 3744ull, 3760ull, 3760ull, 3760ull, 3760ull, 3776ull, 3776ull, 3776ull, 3776ull, 3792ull, 3792ull, 3792ull, 3792ull, 3808ull};
const unsigned kQSubs18[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths18[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs19[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes19[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames19[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs19[] = {3816ull, 3816ull, 3816ull, 3816ull, 3832ull, 3832ull, 3832ull, 3832ull, 3848ull, 3848ull, 3848ull, 3848ull, 3864ull, 3864ull, 3864ull, 3864ull, 3880ull, 3880ull, 3880ull, 3880ull, 3896ull, 3896ull, 3896ull, 3896ull, 3912ull, 3912ull, 3912ull, 3912ull, 3928ull, 3928ull, 3928ull, 3928ull, 3944ull, 3944ull, 3944ull, 3944ull, 3960ull, 3960ull, 3960ull, 3960ull, 3976ull, 3976ull, 3976ull};
const unsigned kQSubs19[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths19[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs20[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 37u, 39u, 40u, 41u, 42u, 43u, 44u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes20[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames20[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs20[] = {3992ull, 3992ull, 3992ull, 3992ull, 4008ull, 4008ull, 4008ull, 4008ull, 4024ull, 4024ull, 4024ull, 4024ull, 4040ull, 4040ull, 4040ull, 4040ull, 4056ull, 4056ull, 4056ull, 4056ull, 4072ull, 4072ull, 4072ull, 4072ull, 4088ull, 4088ull, 4088ull, 4088ull, 4104ull, 4104ull, 4104ull, 4104ull, 4120ull, 4120ull, 4120ull, 4120ull, 4136ull, 4136ull, 4136ull, 4136ull, 4152ull, 4152ull, 4152ull, 4152ull, 4168ull, 4168ull, 4168ull, 4168ull};
const unsigned kQSubs20[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths20[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs21[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 37u, 39u, 40u, 41u, 43u, 44u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes21[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames21[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr11", "vr12", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs21[] = {4192ull, 4192ull, 4192ull, 4192ull, 4208ull, 4208ull, 4208ull, 4208ull, 4224ull, 4224ull, 4224ull, 4224ull, 4240ull, 4240ull, 4240ull, 4240ull, 4256ull, 4256ull, 4256ull, 4256ull, 4272ull, 4272ull, 4272ull, 4272ull, 4288ull, 4288ull, 4288ull, 4288ull, 4304ull, 4304ull, 4304ull, 4304ull, 4320ull, 4320ull, 4320ull, 4320ull, 4336ull, 4336ull, 4336ull, 4336ull, 4352ull, 4352ull, 4352ull, 4352ull, 4368ull, 4368ull, 4368ull};
const unsigned kQSubs21[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths21[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs22[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 37u, 39u, 40u, 41u, 43u, 44u, 57u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes22[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames22[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr11", "vr12", "hit", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs22[] = {4384ull, 4384ull, 4384ull, 4384ull, 4400ull, 4400ull, 4400ull, 4400ull, 4416ull, 4416ull, 4416ull, 4416ull, 4432ull, 4432ull, 4432ull, 4432ull, 4448ull, 4448ull, 4448ull, 4448ull, 4464ull, 4464ull, 4464ull, 4464ull, 4480ull, 4480ull, 4480ull, 4480ull, 4496ull, 4496ull, 4496ull, 4496ull, 4512ull, 4512ull, 4512ull, 4512ull, 4528ull, 4528ull, 4528ull, 4528ull, 4544ull, 4544ull, 4544ull, 4544ull, 4560ull, 4560ull, 4560ull};
const unsigned kQSubs22[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths22[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs23[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 37u, 39u, 40u, 41u, 42u, 43u, 44u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes23[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames23[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs23[] = {4576ull, 4576ull, 4576ull, 4576ull, 4592ull, 4592ull, 4592ull, 4592ull, 4608ull, 4608ull, 4608ull, 4608ull, 4624ull, 4624ull, 4624ull, 4624ull, 4640ull, 4640ull, 4640ull, 4640ull, 4656ull, 4656ull, 4656ull, 4656ull, 4672ull, 4672ull, 4672ull, 4672ull, 4688ull, 4688ull, 4688ull, 4688ull, 4704ull, 4704ull, 4704ull, 4704ull, 4720ull, 4720ull, 4720ull, 4720ull, 4736ull, 4736ull, 4736ull, 4736ull, 4752ull, 4752ull, 4752ull, 4752ull};
const unsigned kQSubs23[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths23[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs24[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 37u, 39u, 40u, 41u, 42u, 43u, 44u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes24[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames24[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs24[] = {4776ull, 4776ull, 4776ull, 4776ull, 4792ull, 4792ull, 4792ull, 4792ull, 4808ull, 4808ull, 4808ull, 4808ull, 4824ull, 4824ull, 4824ull, 4824ull, 4840ull, 4840ull, 4840ull, 4840ull, 4856ull, 4856ull, 4856ull, 4856ull, 4872ull, 4872ull, 4872ull, 4872ull, 4888ull, 4888ull, 4888ull, 4888ull, 4904ull, 4904ull, 4904ull, 4904ull, 4920ull, 4920ull, 4920ull, 4920ull, 4936ull, 4936ull, 4936ull, 4936ull, 4952ull, 4952ull, 4952ull, 4952ull};
const unsigned kQSubs24[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths24[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs25[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 37u, 39u, 40u, 41u, 44u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes25[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames25[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "vr12", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs25[] = {4976ull, 4976ull, 4976ull, 4976ull, 4992ull, 4992ull, 4992ull, 4992ull, 5008ull, 5008ull, 5008ull, 5008ull, 5024ull, 5024ull, 5024ull, 5024ull, 5040ull, 5040ull, 5040ull, 5040ull, 5056ull, 5056ull, 5056ull, 5056ull, 5072ull, 5072ull, 5072ull, 5072ull, 5088ull, 5088ull, 5088ull, 5088ull, 5104ull, 5104ull, 5104ull, 5104ull, 5120ull, 5120ull, 5120ull, 5120ull, 5136ull, 5136ull, 5136ull, 5136ull, 5152ull, 5152ull, 5152ull};
const unsigned kQSubs25[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths25[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs26[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 37u, 39u, 40u, 41u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes26[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames26[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs26[] = {5168ull, 5168ull, 5168ull, 5168ull, 5184ull, 5184ull, 5184ull, 5184ull, 5200ull, 5200ull, 5200ull, 5200ull, 5216ull, 5216ull, 5216ull, 5216ull, 5232ull, 5232ull, 5232ull, 5232ull, 5248ull, 5248ull, 5248ull, 5248ull, 5264ull, 5264ull, 5264ull, 5264ull, 5280ull, 5280ull, 5280ull, 5280ull, 5296ull, 5296ull, 5296ull, 5296ull, 5312ull, 5312ull, 5312ull, 5312ull, 5328ull, 5328ull, 5328ull, 5328ull, 5344ull, 5344ull};
const unsigned kQSubs26[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths26[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs27[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 37u, 39u, 40u, 41u, 57u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes27[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames27[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "hit", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs27[] = {5360ull, 5360ull, 5360ull, 5360ull, 5376ull, 5376ull, 5376ull, 5376ull, 5392ull, 5392ull, 5392ull, 5392ull, 5408ull, 5408ull, 5408ull, 5408ull, 5424ull, 5424ull, 5424ull, 5424ull, 5440ull, 5440ull, 5440ull, 5440ull, 5456ull, 5456ull, 5456ull, 5456ull, 5472ull, 5472ull, 5472ull, 5472ull, 5488ull, 5488ull, 5488ull, 5488ull, 5504ull, 5504ull, 5504ull, 5504ull, 5520ull, 5520ull, 5520ull, 5520ull, 5536ull, 5536ull};
const unsigned kQSubs27[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths27[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs28[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 41u, 57u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes28[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames28[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "hit", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs28[] = {5552ull, 5552ull, 5552ull, 5552ull, 5568ull, 5568ull, 5568ull, 5568ull, 5584ull, 5584ull, 5584ull, 5584ull, 5600ull, 5600ull, 5600ull, 5600ull, 5616ull, 5616ull, 5616ull, 5616ull, 5632ull, 5632ull, 5632ull, 5632ull, 5648ull, 5648ull, 5648ull, 5648ull, 5664ull, 5664ull, 5664ull, 5664ull, 5680ull, 5680ull, 5680ull, 5680ull, 5696ull, 5696ull, 5696ull, 5696ull, 5712ull, 5712ull, 5712ull, 5712ull, 5728ull};
const unsigned kQSubs28[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths28[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs29[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes29[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames29[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs29[] = {5736ull, 5736ull, 5736ull, 5736ull, 5752ull, 5752ull, 5752ull, 5752ull, 5768ull, 5768ull, 5768ull, 5768ull, 5784ull, 5784ull, 5784ull, 5784ull, 5800ull, 5800ull, 5800ull, 5800ull, 5816ull, 5816ull, 5816ull, 5816ull, 5832ull, 5832ull, 5832ull, 5832ull, 5848ull, 5848ull, 5848ull, 5848ull, 5864ull, 5864ull, 5864ull, 5864ull, 5880ull, 5880ull, 5880ull, 5880ull, 5896ull, 5896ull, 5896ull};
const unsigned kQSubs29[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths29[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs30[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 37u, 39u, 40u, 41u, 57u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes30[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames30[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr01", "t", "pid", "rp", "hit", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs30[] = {5912ull, 5912ull, 5912ull, 5912ull, 5928ull, 5928ull, 5928ull, 5928ull, 5944ull, 5944ull, 5944ull, 5944ull, 5960ull, 5960ull, 5960ull, 5960ull, 5976ull, 5976ull, 5976ull, 5976ull, 5992ull, 5992ull, 5992ull, 5992ull, 6008ull, 6008ull, 6008ull, 6008ull, 6024ull, 6024ull, 6024ull, 6024ull, 6040ull, 6040ull, 6040ull, 6040ull, 6056ull, 6056ull, 6056ull, 6056ull, 6072ull, 6072ull, 6072ull, 6072ull, 6088ull, 6088ull};
const unsigned kQSubs30[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths30[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs31[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes31[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames31[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs31[] = {6104ull, 6104ull, 6104ull, 6104ull, 6120ull, 6120ull, 6120ull, 6120ull, 6136ull, 6136ull, 6136ull, 6136ull, 6152ull, 6152ull, 6152ull, 6152ull, 6168ull, 6168ull, 6168ull, 6168ull, 6184ull, 6184ull, 6184ull, 6184ull, 6200ull, 6200ull, 6200ull, 6200ull, 6216ull, 6216ull, 6216ull, 6216ull, 6232ull, 6232ull, 6232ull, 6232ull, 6248ull, 6248ull, 6248ull, 6248ull, 6264ull, 6264ull, 6264ull, 6264ull, 6280ull, 6280ull, 6280ull, 6280ull, 6296ull, 6296ull};
const unsigned kQSubs31[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths31[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs32[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes32[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames32[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs32[] = {6312ull, 6312ull, 6312ull, 6312ull, 6328ull, 6328ull, 6328ull, 6328ull, 6344ull, 6344ull, 6344ull, 6344ull, 6360ull, 6360ull, 6360ull, 6360ull, 6376ull, 6376ull, 6376ull, 6376ull, 6392ull, 6392ull, 6392ull, 6392ull, 6408ull, 6408ull, 6408ull, 6408ull, 6424ull, 6424ull, 6424ull, 6424ull, 6440ull, 6440ull, 6440ull, 6440ull, 6456ull, 6456ull, 6456ull, 6456ull, 6472ull, 6472ull, 6472ull, 6472ull, 6488ull, 6488ull, 6488ull, 6488ull};
const unsigned kQSubs32[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths32[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs33[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 41u, 57u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes33[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames33[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "rp", "hit", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs33[] = {6512ull, 6512ull, 6512ull, 6512ull, 6528ull, 6528ull, 6528ull, 6528ull, 6544ull, 6544ull, 6544ull, 6544ull, 6560ull, 6560ull, 6560ull, 6560ull, 6576ull, 6576ull, 6576ull, 6576ull, 6592ull, 6592ull, 6592ull, 6592ull, 6608ull, 6608ull, 6608ull, 6608ull, 6624ull, 6624ull, 6624ull, 6624ull, 6640ull, 6640ull, 6640ull, 6640ull, 6656ull, 6656ull, 6656ull, 6656ull, 6672ull, 6672ull, 6672ull, 6672ull, 6688ull};
const unsigned kQSubs33[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths33[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs34[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 18u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes34[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames34[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "rpt", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs34[] = {6696ull, 6696ull, 6696ull, 6696ull, 6712ull, 6712ull, 6712ull, 6712ull, 6728ull, 6728ull, 6728ull, 6728ull, 6744ull, 6744ull, 6744ull, 6744ull, 6760ull, 6760ull, 6760ull, 6760ull, 6776ull, 6776ull, 6776ull, 6776ull, 6792ull, 6792ull, 6792ull, 6792ull, 6808ull, 6808ull, 6808ull, 6808ull, 6824ull, 6824ull, 6824ull, 6824ull, 6840ull, 6840ull, 6840ull, 6840ull, 6856ull, 6856ull, 6856ull};
const unsigned kQSubs34[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths34[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs35[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 39u, 40u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes35[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames35[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "t", "pid", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs35[] = {6872ull, 6872ull, 6872ull, 6872ull, 6888ull, 6888ull, 6888ull, 6888ull, 6904ull, 6904ull, 6904ull, 6904ull, 6920ull, 6920ull, 6920ull, 6920ull, 6936ull, 6936ull, 6936ull, 6936ull, 6952ull, 6952ull, 6952ull, 6952ull, 6968ull, 6968ull, 6968ull, 6968ull, 6984ull, 6984ull, 6984ull, 6984ull, 7000ull, 7000ull, 7000ull, 7000ull, 7016ull, 7016ull, 7016ull, 7016ull, 7032ull, 7032ull};
const unsigned kQSubs35[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths35[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs36[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 34u, 35u, 39u, 40u, 61u, 69u, 70u, 71u};
const int kQTypes36[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames36[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "depth", "d2", "t", "pid", "ct", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs36[] = {7048ull, 7048ull, 7048ull, 7048ull, 7064ull, 7064ull, 7064ull, 7064ull, 7080ull, 7080ull, 7080ull, 7080ull, 7096ull, 7096ull, 7096ull, 7096ull, 7112ull, 7112ull, 7112ull, 7112ull, 7128ull, 7128ull, 7128ull, 7128ull, 7144ull, 7144ull, 7144ull, 7144ull, 7160ull, 7160ull, 7160ull, 7160ull};
const unsigned kQSubs36[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths36[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs37[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 40u, 61u, 62u, 63u, 64u, 69u, 70u, 71u};
const int kQTypes37[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames37[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "pid", "ct", "t0", "t1", "t2", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs37[] = {7184ull, 7184ull, 7184ull, 7184ull, 7200ull, 7200ull, 7200ull, 7200ull, 7216ull, 7216ull, 7216ull, 7216ull, 7232ull, 7232ull, 7232ull, 7232ull, 7248ull, 7248ull, 7248ull, 7248ull, 7264ull, 7264ull, 7264ull, 7264ull, 7280ull, 7280ull, 7280ull, 7280ull, 7296ull, 7296ull, 7296ull, 7296ull, 7312ull, 7312ull, 7312ull, 7312ull, 7328ull};
const unsigned kQSubs37[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths37[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs38[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 40u, 61u, 62u, 63u, 64u, 69u, 70u, 71u};
const int kQTypes38[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames38[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "pid", "ct", "t0", "t1", "t2", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs38[] = {7336ull, 7336ull, 7336ull, 7336ull, 7352ull, 7352ull, 7352ull, 7352ull, 7368ull, 7368ull, 7368ull, 7368ull, 7384ull, 7384ull, 7384ull, 7384ull, 7400ull, 7400ull, 7400ull, 7400ull, 7416ull, 7416ull, 7416ull, 7416ull, 7432ull, 7432ull, 7432ull, 7432ull, 7448ull, 7448ull, 7448ull, 7448ull, 7464ull, 7464ull, 7464ull, 7464ull, 7480ull};
const unsigned kQSubs38[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths38[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs39[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 40u, 61u, 62u, 63u, 64u, 69u, 70u, 71u};
const int kQTypes39[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames39[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "pid", "ct", "t0", "t1", "t2", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs39[] = {7488ull, 7488ull, 7488ull, 7488ull, 7504ull, 7504ull, 7504ull, 7504ull, 7520ull, 7520ull, 7520ull, 7520ull, 7536ull, 7536ull, 7536ull, 7536ull, 7552ull, 7552ull, 7552ull, 7552ull, 7568ull, 7568ull, 7568ull, 7568ull, 7584ull, 7584ull, 7584ull, 7584ull, 7600ull, 7600ull, 7600ull, 7600ull, 7616ull, 7616ull, 7616ull, 7616ull, 7632ull};
const unsigned kQSubs39[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths39[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs40[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 40u, 61u, 62u, 63u, 64u, 69u, 70u, 71u};
const int kQTypes40[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames40[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "pid", "ct", "t0", "t1", "t2", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs40[] = {7640ull, 7640ull, 7640ull, 7640ull, 7656ull, 7656ull, 7656ull, 7656ull, 7672ull, 7672ull, 7672ull, 7672ull, 7688ull, 7688ull, 7688ull, 7688ull, 7704ull, 7704ull, 7704ull, 7704ull, 7720ull, 7720ull, 7720ull, 7720ull, 7736ull, 7736ull, 7736ull, 7736ull, 7752ull, 7752ull, 7752ull, 7752ull, 7768ull, 7768ull, 7768ull, 7768ull, 7784ull};
const unsigned kQSubs40[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths40[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs41[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 40u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 69u, 70u, 71u};
const int kQTypes41[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames41[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "pid", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs41[] = {7792ull, 7792ull, 7792ull, 7792ull, 7808ull, 7808ull, 7808ull, 7808ull, 7824ull, 7824ull, 7824ull, 7824ull, 7840ull, 7840ull, 7840ull, 7840ull, 7856ull, 7856ull, 7856ull, 7856ull, 7872ull, 7872ull, 7872ull, 7872ull, 7888ull, 7888ull, 7888ull, 7888ull, 7904ull, 7904ull, 7904ull, 7904ull, 7920ull, 7920ull, 7920ull, 7920ull, 7936ull, 7936ull, 7936ull, 7936ull};
const unsigned kQSubs41[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths41[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs42[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes42[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames42[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs42[] = {7960ull, 7960ull, 7960ull, 7960ull, 7976ull, 7976ull, 7976ull, 7976ull, 7992ull, 7992ull, 7992ull, 7992ull, 8008ull, 8008ull, 8008ull, 8008ull, 8024ull, 8024ull, 8024ull, 8024ull, 8040ull, 8040ull, 8040ull, 8040ull, 8056ull, 8056ull, 8056ull, 8056ull, 8072ull, 8072ull, 8072ull, 8072ull, 8088ull, 8088ull, 8088ull, 8088ull, 8104ull, 8104ull, 8104ull, 8104ull, 8120ull};
const unsigned kQSubs42[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths42[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs43[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 21u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u};
const int kQTypes43[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames43[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "u1", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal"};
const unsigned long long kQOffs43[] = {8128ull, 8128ull, 8128ull, 8128ull, 8144ull, 8144ull, 8144ull, 8144ull, 8160ull, 8160ull, 8160ull, 8160ull, 8176ull, 8176ull, 8176ull, 8176ull, 8192ull, 8192ull, 8192ull, 8192ull, 8208ull, 8208ull, 8208ull, 8208ull, 8224ull, 8224ull, 8224ull, 8224ull, 8240ull, 8240ull, 8240ull, 8240ull, 8256ull, 8256ull, 8256ull, 8256ull, 8272ull, 8272ull, 8272ull};
const unsigned kQSubs43[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths43[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs44[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 40u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes44[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames44[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "pid", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs44[] = {8288ull, 8288ull, 8288ull, 8288ull, 8304ull, 8304ull, 8304ull, 8304ull, 8320ull, 8320ull, 8320ull, 8320ull, 8336ull, 8336ull, 8336ull, 8336ull, 8352ull, 8352ull, 8352ull, 8352ull, 8368ull, 8368ull, 8368ull, 8368ull, 8384ull, 8384ull, 8384ull, 8384ull, 8400ull, 8400ull, 8400ull, 8400ull, 8416ull, 8416ull, 8416ull, 8416ull, 8432ull, 8432ull, 8432ull, 8432ull, 8448ull};
const unsigned kQSubs44[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths44[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs45[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes45[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames45[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "tmp1", "tmp2", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs45[] = {8456ull, 8456ull, 8456ull, 8456ull, 8472ull, 8472ull, 8472ull, 8472ull, 8488ull, 8488ull, 8488ull, 8488ull, 8504ull, 8504ull, 8504ull, 8504ull, 8520ull, 8520ull, 8520ull, 8520ull, 8536ull, 8536ull, 8536ull, 8536ull, 8552ull, 8552ull, 8552ull, 8552ull, 8568ull, 8568ull, 8568ull, 8568ull, 8584ull, 8584ull, 8584ull, 8584ull, 8600ull, 8600ull, 8600ull, 8600ull, 8616ull, 8616ull};
const unsigned kQSubs45[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths45[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs46[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 21u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes46[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames46[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "u1", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs46[] = {8632ull, 8632ull, 8632ull, 8632ull, 8648ull, 8648ull, 8648ull, 8648ull, 8664ull, 8664ull, 8664ull, 8664ull, 8680ull, 8680ull, 8680ull, 8680ull, 8696ull, 8696ull, 8696ull, 8696ull, 8712ull, 8712ull, 8712ull, 8712ull, 8728ull, 8728ull, 8728ull, 8728ull, 8744ull, 8744ull, 8744ull, 8744ull, 8760ull, 8760ull, 8760ull, 8760ull, 8776ull, 8776ull, 8776ull, 8776ull, 8792ull, 8792ull};
const unsigned kQSubs46[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths46[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs47[] = {1u, 2u, 3u, 4u, 5u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 21u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 61u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes47[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames47[] = {"ppp", "L0", "L1", "L2", "rc", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "u1", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "ct", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs47[] = {8808ull, 8808ull, 8808ull, 8808ull, 8824ull, 8824ull, 8824ull, 8824ull, 8840ull, 8840ull, 8840ull, 8840ull, 8856ull, 8856ull, 8856ull, 8856ull, 8872ull, 8872ull, 8872ull, 8872ull, 8888ull, 8888ull, 8888ull, 8888ull, 8904ull, 8904ull, 8904ull, 8904ull, 8920ull, 8920ull, 8920ull, 8920ull, 8936ull, 8936ull, 8936ull, 8936ull};
const unsigned kQSubs47[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths47[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs48[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes48[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames48[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs48[] = {8960ull, 8960ull, 8960ull, 8960ull, 8976ull, 8976ull, 8976ull, 8976ull, 8992ull, 8992ull, 8992ull, 8992ull, 9008ull, 9008ull, 9008ull, 9008ull, 9024ull, 9024ull, 9024ull, 9024ull, 9040ull, 9040ull, 9040ull, 9040ull, 9056ull, 9056ull, 9056ull, 9056ull, 9072ull, 9072ull, 9072ull, 9072ull, 9088ull, 9088ull, 9088ull, 9088ull, 9104ull, 9104ull, 9104ull, 9104ull, 9120ull};
const unsigned kQSubs48[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths48[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs49[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes49[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames49[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs49[] = {9128ull, 9128ull, 9128ull, 9128ull, 9144ull, 9144ull, 9144ull, 9144ull, 9160ull, 9160ull, 9160ull, 9160ull, 9176ull, 9176ull, 9176ull, 9176ull, 9192ull, 9192ull, 9192ull, 9192ull, 9208ull, 9208ull, 9208ull, 9208ull, 9224ull, 9224ull, 9224ull, 9224ull, 9240ull, 9240ull, 9240ull, 9240ull, 9256ull, 9256ull, 9256ull, 9256ull, 9272ull, 9272ull};
const unsigned kQSubs49[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths49[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs50[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 21u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes50[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames50[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "u1", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs50[] = {9288ull, 9288ull, 9288ull, 9288ull, 9304ull, 9304ull, 9304ull, 9304ull, 9320ull, 9320ull, 9320ull, 9320ull, 9336ull, 9336ull, 9336ull, 9336ull, 9352ull, 9352ull, 9352ull, 9352ull, 9368ull, 9368ull, 9368ull, 9368ull, 9384ull, 9384ull, 9384ull, 9384ull, 9400ull, 9400ull, 9400ull, 9400ull, 9416ull, 9416ull, 9416ull, 9416ull, 9432ull, 9432ull, 9432ull, 9432ull, 9448ull, 9448ull};
const unsigned kQSubs50[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths50[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs51[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 20u, 21u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes51[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames51[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "u0", "u1", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "vr02", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs51[] = {9464ull, 9464ull, 9464ull, 9464ull, 9480ull, 9480ull, 9480ull, 9480ull, 9496ull, 9496ull, 9496ull, 9496ull, 9512ull, 9512ull, 9512ull, 9512ull, 9528ull, 9528ull, 9528ull, 9528ull, 9544ull, 9544ull, 9544ull, 9544ull, 9560ull, 9560ull, 9560ull, 9560ull, 9576ull, 9576ull, 9576ull, 9576ull, 9592ull, 9592ull, 9592ull, 9592ull, 9608ull, 9608ull, 9608ull, 9608ull, 9624ull, 9624ull, 9624ull, 9624ull, 9640ull};
const unsigned kQSubs51[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths51[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs52[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 10u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes52[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames52[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "tmp1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "vr00", "vr01", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs52[] = {9648ull, 9648ull, 9648ull, 9648ull, 9664ull, 9664ull, 9664ull, 9664ull, 9680ull, 9680ull, 9680ull, 9680ull, 9696ull, 9696ull, 9696ull, 9696ull, 9712ull, 9712ull, 9712ull, 9712ull, 9728ull, 9728ull, 9728ull, 9728ull, 9744ull, 9744ull, 9744ull, 9744ull, 9760ull, 9760ull, 9760ull, 9760ull, 9776ull, 9776ull, 9776ull, 9776ull, 9792ull, 9792ull, 9792ull, 9792ull, 9808ull, 9808ull, 9808ull, 9808ull};
const unsigned kQSubs52[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths52[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs53[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 10u, 11u, 12u, 13u, 15u, 16u, 17u, 19u, 22u, 23u, 24u, 25u, 26u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 61u, 62u, 63u, 64u, 65u, 66u, 67u, 68u, 69u, 70u, 71u};
const int kQTypes53[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames53[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "mean", "m2", "ns", "o0", "o1", "o2", "TP0", "TP1", "TP2", "SL0", "SL1", "SL2", "clr0", "clr1", "clr2", "depth", "d2", "ct", "t0", "t1", "t2", "n0", "n1", "n2", "metal", "wi0", "wi1", "wi2"};
const unsigned long long kQOffs53[] = {9832ull, 9832ull, 9832ull, 9832ull, 9848ull, 9848ull, 9848ull, 9848ull, 9864ull, 9864ull, 9864ull, 9864ull, 9880ull, 9880ull, 9880ull, 9880ull, 9896ull, 9896ull, 9896ull, 9896ull, 9912ull, 9912ull, 9912ull, 9912ull, 9928ull, 9928ull, 9928ull, 9928ull, 9944ull, 9944ull, 9944ull, 9944ull, 9960ull, 9960ull, 9960ull, 9960ull, 9976ull, 9976ull, 9976ull, 9976ull};
const unsigned kQSubs53[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths53[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs54[] = {1u, 2u, 3u, 4u, 5u, 19u};
const int kQTypes54[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames54[] = {"ppp", "L0", "L1", "L2", "rc", "ns"};
const unsigned long long kQOffs54[] = {10000ull, 10000ull, 10000ull, 10000ull, 10016ull, 10016ull};
const unsigned kQSubs54[] = {0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths54[] = {16u, 16u, 16u, 16u, 16u, 16u};
const loom_b200_queue_layout kQueues[] = {
    {0u, -1, 27u, kQRegs0, kQTypes0, kQNames0},
    {1u, -1, 41u, kQRegs1, kQTypes1, kQNames1},
    {2u, -1, 45u, kQRegs2, kQTypes2, kQNames2},
    {3u, -1, 27u, kQRegs3, kQTypes3, kQNames3},
    {4u, -1, 41u, kQRegs4, kQTypes4, kQNames4},
    {5u, -1, 44u, kQRegs5, kQTypes5, kQNames5},
    {6u, -1, 60u, kQRegs6, kQTypes6, kQNames6},
    {7u, -1, 58u, kQRegs7, kQTypes7, kQNames7},
    {8u, -1, 58u, kQRegs8, kQTypes8, kQNames8},
    {9u, -1, 56u, kQRegs9, kQTypes9, kQNames9},
    {10u, -1, 63u, kQRegs10, kQTypes10, kQNames10},
    {11u, -1, 60u, kQRegs11, kQTypes11, kQNames11},
    {12u, -1, 53u, kQRegs12, kQTypes12, kQNames12},
    {13u, -1, 45u, kQRegs13, kQTypes13, kQNames13},
    {14u, -1, 43u, kQRegs14, kQTypes14, kQNames14},
    {15u, -1, 56u, kQRegs15, kQTypes15, kQNames15},
    {16u, -1, 54u, kQRegs16, kQTypes16, kQNames16},
    {17u, -1, 50u, kQRegs17, kQTypes17, kQNames17},
    {18u, -1, 45u, kQRegs18, kQTypes18, kQNames18},
    {19u, -1, 43u, kQRegs19, kQTypes19, kQNames19},
    {20u, -1, 48u, kQRegs20, kQTypes20, kQNames20},
    {21u, -1, 47u, kQRegs21, kQTypes21, kQNames21},
    {22u, -1, 47u, kQRegs22, kQTypes22, kQNames22},
    {23u, -1, 48u, kQRegs23, kQTypes23, kQNames23},
    {24u, -1, 48u, kQRegs24, kQTypes24, kQNames24},
    {25u, -1, 47u, kQRegs25, kQTypes25, kQNames25},
    {26u, -1, 46u, kQRegs26, kQTypes26, kQNames26},
    {27u, -1, 46u, kQRegs27, kQTypes27, kQNames27},
    {28u, -1, 45u, kQRegs28, kQTypes28, kQNames28},
    {29u, -1, 43u, kQRegs29, kQTypes29, kQNames29},
    {30u, -1, 46u, kQRegs30, kQTypes30, kQNames30},
    {31u, -1, 50u, kQRegs31, kQTypes31, kQNames31},
    {32u, -1, 48u, kQRegs32, kQTypes32, kQNames32},
    {33u, -1, 45u, kQRegs33, kQTypes33, kQNames33},
    {34u, -1, 43u, kQRegs34, kQTypes34, kQNames34},
    {35u, -1, 42u, kQRegs35, kQTypes35, kQNames35},
    {36u, -1, 32u, kQRegs36, kQTypes36, kQNames36},
    {37u, -1, 37u, kQRegs37, kQTypes37, kQNames37},
    {38u, -1, 37u, kQRegs38, kQTypes38, kQNames38},
    {39u, -1, 37u, kQRegs39, kQTypes39, kQNames39},
    {40u, -1, 37u, kQRegs40, kQTypes40, kQNames40},
    {41u, -1, 40u, kQRegs41, kQTypes41, kQNames41},
    {42u, -1, 41u, kQRegs42, kQTypes42, kQNames42},
    {43u, -1, 39u, kQRegs43, kQTypes43, kQNames43},
    {44u, -1, 41u, kQRegs44, kQTypes44, kQNames44},
    {45u, -1, 42u, kQRegs45, kQTypes45, kQNames45},
    {46u, -1, 42u, kQRegs46, kQTypes46, kQNames46},
    {47u, -1, 36u, kQRegs47, kQTypes47, kQNames47},
    {48u, -1, 41u, kQRegs48, kQTypes48, kQNames48},
    {49u, -1, 38u, kQRegs49, kQTypes49, kQNames49},
    {50u, -1, 42u, kQRegs50, kQTypes50, kQNames50},
    {51u, -1, 45u, kQRegs51, kQTypes51, kQNames51},
    {52u, -1, 44u, kQRegs52, kQTypes52, kQNames52},
    {53u, -1, 40u, kQRegs53, kQTypes53, kQNames53},
    {54u, -1, 6u, kQRegs54, kQTypes54, kQNames54},
};
const QueueSegment kSegments[] = {
    {kQOffs0, kQSubs0, kQWidths0, 96ull, 12u, 16u},
    {kQOffs1, kQSubs1, kQWidths1, 272ull, 4u, 8u},
    {kQOffs2, kQSubs2, kQWidths2, 456ull, 4u, 8u},
    {kQOffs3, kQSubs3, kQWidths3, 560ull, 12u, 16u},
    {kQOffs4, kQSubs4, kQWidths4, 736ull, 4u, 8u},
    {kQOffs5, kQSubs5, kQWidths5, 920ull, 0u, 4u},
    {kQOffs6, kQSubs6, kQWidths6, 1168ull, 0u, 4u},
    {kQOffs7, kQSubs7, kQWidths7, 1400ull, 8u, 16u},
    {kQOffs8, kQSubs8, kQWidths8, 1640ull, 8u, 16u},
    {kQOffs9, kQSubs9, kQWidths9, 1880ull, 0u, 4u},
    {kQOffs10, kQSubs10, kQWidths10, 2128ull, 12u, 16u},
    {kQOffs11, kQSubs11, kQWidths11, 2384ull, 0u, 4u},
    {kQOffs12, kQSubs12, kQWidths12, 2600ull, 4u, 8u},
    {kQOffs13, kQSubs13, kQWidths13, 2784ull, 4u, 8u},
    {kQOffs14, kQSubs14, kQWidths14, 2952ull, 12u, 16u},
    {kQOffs15, kQSubs15, kQWidths15, 3192ull, 0u, 4u},
    {kQOffs16, kQSubs16, kQWidths16, 3408ull, 8u, 16u},
    {kQOffs17, kQSubs17, kQWidths17, 3616ull, 8u, 16u},
    {kQOffs18, kQSubs18, kQWidths18, 3808ull, 4u, 8u},
    {kQOffs19, kQSubs19, kQWidths19, 3976ull, 12u, 16u},
    {kQOffs20, kQSubs20, kQWidths20, 4184ull, 0u, 4u},
    {kQOffs21, kQSubs21, kQWidths21, 4368ull, 12u, 16u},
    {kQOffs22, kQSubs22, kQWidths22, 4560ull, 12u, 16u},
    {kQOffs23, kQSubs23, kQWidths23, 4768ull, 0u, 4u},
    {kQOffs24, kQSubs24, kQWidths24, 4968ull, 0u, 4u},
    {kQOffs25, kQSubs25, kQWidths25, 5152ull, 12u, 16u},
    {kQOffs26, kQSubs26, kQWidths26, 5344ull, 8u, 16u},
    {kQOffs27, kQSubs27, kQWidths27, 5536ull, 8u, 16u},
    {kQOffs28, kQSubs28, kQWidths28, 5728ull, 4u, 8u},
    {kQOffs29, kQSubs29, kQWidths29, 5896ull, 12u, 16u},
    {kQOffs30, kQSubs30, kQWidths30, 6088ull, 8u, 16u},
    {kQOffs31, kQSubs31, kQWidths31, 6296ull, 8u, 16u},
    {kQOffs32, kQSubs32, kQWidths32, 6504ull, 0u, 4u},
    {kQOffs33, kQSubs33, kQWidths33, 6688ull, 4u, 8u},
    {kQOffs34, kQSubs34, kQWidths34, 6856ull, 12u, 16u},
    {kQOffs35, kQSubs35, kQWidths35, 7032ull, 8u, 16u},
    {kQOffs36, kQSubs36, kQWidths36, 7176ull, 0u, 4u},
    {kQOffs37, kQSubs37, kQWidths37, 7328ull, 4u, 8u},
    {kQOffs38, kQSubs38, kQWidths38, 7480ull, 4u, 8u},
    {kQOffs39, kQSubs39, kQWidths39, 7632ull, 4u, 8u},
    {kQOffs40, kQSubs40, kQWidths40, 7784ull, 4u, 8u},
    {kQOffs41, kQSubs41, kQWidths41, 7952ull, 0u, 4u},
    {kQOffs42, kQSubs42, kQWidths42, 8120ull, 4u, 8u},
    {kQOffs43, kQSubs43, kQWidths43, 8272ull, 12u, 16u},
    {kQOffs44, kQSubs44, kQWidths44, 8448ull, 4u, 8u},
    {kQOffs45, kQSubs45, kQWidths45, 8616ull, 8u, 16u},
    {kQOffs46, kQSubs46, kQWidths46, 8792ull, 8u, 16u},
    {kQOffs47, kQSubs47, kQWidths47, 8952ull, 0u, 4u},
    {kQOffs48, kQSubs48, kQWidths48, 9120ull, 4u, 8u},
    {kQOffs49, kQSubs49, kQWidths49, 9272ull, 8u, 16u},
    {kQOffs50, kQSubs50, kQWidths50, 9448ull, 8u, 16u},
    {kQOffs51, kQSubs51, kQWidths51, 9640ull, 4u, 8u},
    {kQOffs52, kQSubs52, kQWidths52, 9824ull, 0u, 4u},
    {kQOffs53, kQSubs53, kQWidths53, 9992ull, 0u, 4u},
    {kQOffs54, kQSubs54, kQWidths54, 10016ull, 8u, 16u},
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

} } // namespace loom_b200::k_pt2_const_512

extern const loom_b200::KernelEntry loom_b200_entry_pt2_const_512;
const loom_b200::KernelEntry loom_b200_entry_pt2_const_512 = {
    &loom_b200::k_pt2_const_512::kInfo, loom_b200::k_pt2_const_512::K::kRowBytes, 55,
    &loom_b200::k_pt2_const_512::launch_plain, &loom_b200::k_pt2_const_512::launch_regroup,
    &loom_b200::k_pt2_const_512::regroup_occupancy,
    loom_b200::k_pt2_const_512::kQueues, loom_b200::k_pt2_const_512::kSegments,
    loom_b200::k_pt2_const_512::kRegCaps, 8u, loom_b200::k_pt2_const_512::K::kMaxStageRow};
