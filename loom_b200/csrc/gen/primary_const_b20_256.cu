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
            reinterpret_cast<unsigned int*>(base + 0ull * cap)[idx] = R.r1;
            reinterpret_cast<unsigned int*>(base + 4ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 8ull * cap)[idx] = tid;
            return;
        case 1: // roll
            reinterpret_cast<unsigned int*>(base + 16ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 20ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 24ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 28ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 32ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 36ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 40ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 44ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 48ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 52ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 56ull * cap)[idx] = R.r17;
            reinterpret_cast<unsigned int*>(base + 60ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 64ull * cap)[idx] = tid;
            return;
        case 2: // traverse_box
            reinterpret_cast<unsigned int*>(base + 72ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 76ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 80ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 84ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 88ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 92ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 96ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 100ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 104ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 108ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 112ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 116ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 120ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 124ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 128ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 132ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 136ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 140ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 144ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 148ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 152ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 156ull * cap)[idx] = tid;
            return;
        case 3: // isect_quad_l1
            reinterpret_cast<unsigned int*>(base + 160ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 164ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 168ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 172ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 176ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 180ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 184ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 188ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 192ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 196ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 200ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 204ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 208ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 212ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 216ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 220ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 224ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 228ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 232ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 236ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 240ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 244ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 248ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 252ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 256ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 260ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 264ull * cap)[idx] = R.r36;
            reinterpret_cast<float*>(base + 268ull * cap)[idx] = R.r37;
            reinterpret_cast<float*>(base + 272ull * cap)[idx] = R.r38;
            reinterpret_cast<float*>(base + 276ull * cap)[idx] = R.r39;
            reinterpret_cast<float*>(base + 280ull * cap)[idx] = R.r40;
            reinterpret_cast<float*>(base + 284ull * cap)[idx] = R.r41;
            reinterpret_cast<float*>(base + 288ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 292ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 296ull * cap)[idx] = R.r51;
            reinterpret_cast<float*>(base + 300ull * cap)[idx] = R.r52;
            reinterpret_cast<unsigned int*>(base + 304ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 308ull * cap)[idx] = tid;
            return;
        case 4: // isect_quad_l2
            reinterpret_cast<unsigned int*>(base + 312ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 316ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 320ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 324ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 328ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 332ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 336ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 340ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 344ull * cap)[idx] = R.r9;
            reinterpret_cast<unsigned int*>(base + 348ull * cap)[idx] = R.r10;
            reinterpret_cast<float*>(base + 352ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 356ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 360ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 364ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 368ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 372ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 376ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 380ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 384ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 388ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 392ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 396ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 400ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 404ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 408ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 412ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 416ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 420ull * cap)[idx] = R.r36;
            reinterpret_cast<float*>(base + 424ull * cap)[idx] = R.r37;
            reinterpret_cast<float*>(base + 428ull * cap)[idx] = R.r38;
            reinterpret_cast<float*>(base + 432ull * cap)[idx] = R.r39;
            reinterpret_cast<float*>(base + 436ull * cap)[idx] = R.r40;
            reinterpret_cast<float*>(base + 440ull * cap)[idx] = R.r41;
            reinterpret_cast<float*>(base + 444ull * cap)[idx] = R.r42;
            reinterpret_cast<unsigned int*>(base + 448ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 452ull * cap)[idx] = tid;
            return;
        case 5: // isect_quad_l3
            reinterpret_cast<unsigned int*>(base + 456ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 460ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 464ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 468ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 472ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 476ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 480ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 484ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 488ull * cap)[idx] = R.r9;
            reinterpret_cast<unsigned int*>(base + 492ull * cap)[idx] = R.r10;
            reinterpret_cast<unsigned int*>(base + 496ull * cap)[idx] = R.r11;
            reinterpret_cast<float*>(base + 500ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 504ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 508ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 512ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 516ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 520ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 524ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 528ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 532ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 536ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 540ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 544ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 548ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 552ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 556ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 560ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 564ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 568ull * cap)[idx] = R.r36;
            reinterpret_cast<float*>(base + 572ull * cap)[idx] = R.r37;
            reinterpret_cast<float*>(base + 576ull * cap)[idx] = R.r38;
            reinterpret_cast<float*>(base + 580ull * cap)[idx] = R.r39;
            reinterpret_cast<float*>(base + 584ull * cap)[idx] = R.r40;
            reinterpret_cast<float*>(base + 588ull * cap)[idx] = R.r41;
            reinterpret_cast<float*>(base + 592ull * cap)[idx] = R.r42;
            reinterpret_cast<unsigned*>(base + 596ull * cap)[idx] = tid;
            return;
        case 6: // isect_quad_l4
            reinterpret_cast<unsigned int*>(base + 600ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 604ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 608ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 612ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 616ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 620ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 624ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 628ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 632ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 636ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 640ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 644ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 648ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 652ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 656ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 660ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 664ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 668ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 672ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 676ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 680ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 684ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 688ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 692ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 696ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 700ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 704ull * cap)[idx] = R.r36;
            reinterpret_cast<float*>(base + 708ull * cap)[idx] = R.r37;
            reinterpret_cast<float*>(base + 712ull * cap)[idx] = R.r38;
            reinterpret_cast<float*>(base + 716ull * cap)[idx] = R.r39;
            reinterpret_cast<float*>(base + 720ull * cap)[idx] = R.r40;
            reinterpret_cast<float*>(base + 724ull * cap)[idx] = R.r41;
            reinterpret_cast<float*>(base + 728ull * cap)[idx] = R.r42;
            reinterpret_cast<unsigned*>(base + 732ull * cap)[idx] = tid;
            return;
        case 7: // isect_quad_l5
            reinterpret_cast<unsigned int*>(base + 736ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 740ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 744ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 748ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 752ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 756ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 760ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 764ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 768ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 772ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 776ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 780ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 784ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 788ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 792ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 796ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 800ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 804ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 808ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 812ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 816ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 820ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 824ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 828ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 832ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 836ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 840ull * cap)[idx] = R.r36;
            reinterpret_cast<float*>(base + 844ull * cap)[idx] = R.r37;
            reinterpret_cast<float*>(base + 848ull * cap)[idx] = R.r38;
            reinterpret_cast<float*>(base + 852ull * cap)[idx] = R.r39;
            reinterpret_cast<float*>(base + 856ull * cap)[idx] = R.r40;
            reinterpret_cast<float*>(base + 860ull * cap)[idx] = R.r41;
            reinterpret_cast<float*>(base + 864ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 868ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 872ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 876ull * cap)[idx] = R.r45;
            reinterpret_cast<float*>(base + 880ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 884ull * cap)[idx] = R.r51;
            reinterpret_cast<float*>(base + 888ull * cap)[idx] = R.r52;
            reinterpret_cast<unsigned int*>(base + 892ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 896ull * cap)[idx] = tid;
            return;
        case 8: // isect_quad_l6
            reinterpret_cast<unsigned int*>(base + 904ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 908ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 912ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 916ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 920ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 924ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 928ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 932ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 936ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 940ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 944ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 948ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 952ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 956ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 960ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 964ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 968ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 972ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 976ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 980ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 984ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 988ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 992ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 996ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 1000ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 1004ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 1008ull * cap)[idx] = R.r36;
            reinterpret_cast<float*>(base + 1012ull * cap)[idx] = R.r40;
            reinterpret_cast<float*>(base + 1016ull * cap)[idx] = R.r41;
            reinterpret_cast<float*>(base + 1020ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 1024ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 1028ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 1032ull * cap)[idx] = R.r45;
            reinterpret_cast<float*>(base + 1036ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 1040ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 1044ull * cap)[idx] = R.r48;
            reinterpret_cast<unsigned int*>(base + 1048ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 1052ull * cap)[idx] = tid;
            return;
        case 9: // isect_quad_l7
            reinterpret_cast<unsigned int*>(base + 1056ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 1060ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 1064ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1068ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 1072ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1076ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 1080ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 1084ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 1088ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 1092ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 1096ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1100ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 1104ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 1108ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 1112ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 1116ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 1120ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 1124ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 1128ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 1132ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 1136ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 1140ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 1144ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 1148ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 1152ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 1156ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 1160ull * cap)[idx] = R.r36;
            reinterpret_cast<float*>(base + 1164ull * cap)[idx] = R.r40;
            reinterpret_cast<float*>(base + 1168ull * cap)[idx] = R.r41;
            reinterpret_cast<float*>(base + 1172ull * cap)[idx] = R.r42;
            reinterpret_cast<unsigned*>(base + 1176ull * cap)[idx] = tid;
            return;
        case 10: // isect_quad_end
            reinterpret_cast<unsigned int*>(base + 1184ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 1188ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 1192ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1196ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 1200ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1204ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 1208ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 1212ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 1216ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 1220ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 1224ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 1228ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 1232ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 1236ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 1240ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 1244ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 1248ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 1252ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 1256ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 1260ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 1264ull * cap)[idx] = R.r49;
            reinterpret_cast<unsigned int*>(base + 1268ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 1272ull * cap)[idx] = tid;
            return;
        case 11: // traverse_tetrahedron
            reinterpret_cast<unsigned int*>(base + 1280ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 1284ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 1288ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1292ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 1296ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1300ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 1304ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 1308ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 1312ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 1316ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 1320ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 1324ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 1328ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 1332ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 1336ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 1340ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 1344ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 1348ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 1352ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 1356ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned*>(base + 1360ull * cap)[idx] = tid;
            return;
        case 12: // isect_triangle_mid1
            reinterpret_cast<unsigned int*>(base + 1368ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 1372ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 1376ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1380ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 1384ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1388ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 1392ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 1396ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 1400ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 1404ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 1408ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 1412ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 1416ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 1420ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 1424ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 1428ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 1432ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 1436ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 1440ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 1444ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 1448ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 1452ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 1456ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 1460ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 1464ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 1468ull * cap)[idx] = R.r36;
            reinterpret_cast<float*>(base + 1472ull * cap)[idx] = R.r37;
            reinterpret_cast<float*>(base + 1476ull * cap)[idx] = R.r38;
            reinterpret_cast<float*>(base + 1480ull * cap)[idx] = R.r39;
            reinterpret_cast<float*>(base + 1484ull * cap)[idx] = R.r40;
            reinterpret_cast<float*>(base + 1488ull * cap)[idx] = R.r41;
            reinterpret_cast<float*>(base + 1492ull * cap)[idx] = R.r42;
            reinterpret_cast<unsigned int*>(base + 1496ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 1500ull * cap)[idx] = tid;
            return;
        case 13: // isect_triangle_mid2
            reinterpret_cast<unsigned int*>(base + 1504ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 1508ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 1512ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1516ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 1520ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1524ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 1528ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 1532ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 1536ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 1540ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 1544ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1548ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 1552ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 1556ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 1560ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 1564ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 1568ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 1572ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 1576ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 1580ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 1584ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 1588ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 1592ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 1596ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 1600ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 1604ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 1608ull * cap)[idx] = R.r36;
            reinterpret_cast<float*>(base + 1612ull * cap)[idx] = R.r37;
            reinterpret_cast<float*>(base + 1616ull * cap)[idx] = R.r38;
            reinterpret_cast<float*>(base + 1620ull * cap)[idx] = R.r39;
            reinterpret_cast<unsigned int*>(base + 1624ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 1628ull * cap)[idx] = tid;
            return;
        case 14: // isect_triangle_mid3
            reinterpret_cast<unsigned int*>(base + 1632ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 1636ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 1640ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1644ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 1648ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1652ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 1656ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 1660ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 1664ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 1668ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 1672ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 1676ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 1680ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 1684ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 1688ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 1692ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 1696ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 1700ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 1704ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 1708ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 1712ull * cap)[idx] = R.r37;
            reinterpret_cast<float*>(base + 1716ull * cap)[idx] = R.r38;
            reinterpret_cast<float*>(base + 1720ull * cap)[idx] = R.r39;
            reinterpret_cast<float*>(base + 1724ull * cap)[idx] = R.r40;
            reinterpret_cast<float*>(base + 1728ull * cap)[idx] = R.r41;
            reinterpret_cast<float*>(base + 1732ull * cap)[idx] = R.r42;
            reinterpret_cast<unsigned int*>(base + 1736ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 1740ull * cap)[idx] = tid;
            return;
        case 15: // isect_triangle_end
            reinterpret_cast<unsigned int*>(base + 1744ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 1748ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 1752ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1756ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 1760ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1764ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 1768ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 1772ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 1776ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 1780ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 1784ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 1788ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 1792ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 1796ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 1800ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 1804ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 1808ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 1812ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 1816ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 1820ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 1824ull * cap)[idx] = R.r49;
            reinterpret_cast<unsigned int*>(base + 1828ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 1832ull * cap)[idx] = tid;
            return;
        case 16: // traverse_sphere
            reinterpret_cast<unsigned int*>(base + 1840ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 1844ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 1848ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1852ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 1856ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1860ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 1864ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 1868ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 1872ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 1876ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 1880ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 1884ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 1888ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 1892ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 1896ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 1900ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 1904ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 1908ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 1912ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 1916ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 1920ull * cap)[idx] = tid;
            return;
        case 17: // traverse_solve_quadratic
            reinterpret_cast<unsigned int*>(base + 1928ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 1932ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 1936ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1940ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 1944ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1948ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 1952ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 1956ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 1960ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 1964ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 1968ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 1972ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 1976ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 1980ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 1984ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 1988ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 1992ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 1996ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 2000ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2004ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2008ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 2012ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 2016ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 2020ull * cap)[idx] = R.r36;
            reinterpret_cast<unsigned int*>(base + 2024ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 2028ull * cap)[idx] = tid;
            return;
        case 18: // sq_head1
            reinterpret_cast<unsigned int*>(base + 2032ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2036ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2040ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2044ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2048ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2052ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2056ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2060ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2064ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2068ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2072ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 2076ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2080ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2084ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2088ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2092ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2096ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2100ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 2104ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2108ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2112ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 2116ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 2120ull * cap)[idx] = R.r36;
            reinterpret_cast<unsigned int*>(base + 2124ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 2128ull * cap)[idx] = tid;
            return;
        case 19: // sq_head2
            reinterpret_cast<unsigned int*>(base + 2136ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2140ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2144ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2148ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2152ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2156ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2160ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2164ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2168ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2172ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2176ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 2180ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2184ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2188ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2192ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2196ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2200ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2204ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 2208ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2212ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2216ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 2220ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 2224ull * cap)[idx] = R.r36;
            reinterpret_cast<unsigned int*>(base + 2228ull * cap)[idx] = R.r49;
            reinterpret_cast<unsigned*>(base + 2232ull * cap)[idx] = tid;
            return;
        case 20: // sq_mid1
            reinterpret_cast<unsigned int*>(base + 2240ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2244ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2248ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2252ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2256ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2260ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2264ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2268ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2272ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2276ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2280ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 2284ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2288ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2292ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2296ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2300ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2304ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2308ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 2312ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2316ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2320ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 2324ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 2328ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 2332ull * cap)[idx] = R.r36;
            reinterpret_cast<unsigned int*>(base + 2336ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 2340ull * cap)[idx] = tid;
            return;
        case 21: // sq_mid2
            reinterpret_cast<unsigned int*>(base + 2344ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2348ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2352ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2356ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2360ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2364ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2368ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2372ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2376ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2380ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2384ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 2388ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 2392ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2396ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2400ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2404ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2408ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2412ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2416ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 2420ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2424ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2428ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 2432ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 2436ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 2440ull * cap)[idx] = R.r36;
            reinterpret_cast<unsigned*>(base + 2444ull * cap)[idx] = tid;
            return;
        case 22: // sq_mid
            reinterpret_cast<unsigned int*>(base + 2448ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2452ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2456ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2460ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2464ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2468ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2472ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2476ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2480ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2484ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2488ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 2492ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 2496ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2500ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2504ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2508ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2512ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2516ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2520ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 2524ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2528ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2532ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 2536ull * cap)[idx] = R.r36;
            reinterpret_cast<unsigned int*>(base + 2540ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 2544ull * cap)[idx] = tid;
            return;
        case 23: // sq_tail
            reinterpret_cast<unsigned int*>(base + 2552ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2556ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2560ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2564ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2568ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2572ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2576ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2580ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2584ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2588ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2592ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 2596ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 2600ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2604ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2608ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2612ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2616ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2620ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2624ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 2628ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2632ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2636ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 2640ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 2644ull * cap)[idx] = tid;
            return;
        case 24: // sq_end
            reinterpret_cast<unsigned int*>(base + 2648ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2652ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2656ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2660ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2664ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2668ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2672ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2676ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2680ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2684ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2688ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 2692ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2696ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2700ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2704ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2708ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2712ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2716ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 2720ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2724ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2728ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 2732ull * cap)[idx] = R.r49;
            reinterpret_cast<unsigned int*>(base + 2736ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 2740ull * cap)[idx] = tid;
            return;
        case 25: // traverse_sphere_fin
            reinterpret_cast<unsigned int*>(base + 2744ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2748ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2752ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2756ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2760ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2764ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2768ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2772ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2776ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2780ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2784ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 2788ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2792ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2796ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2800ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2804ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2808ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2812ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2816ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2820ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 2824ull * cap)[idx] = R.r49;
            reinterpret_cast<unsigned int*>(base + 2828ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 2832ull * cap)[idx] = tid;
            return;
        case 26: // traverse_cylinder
            reinterpret_cast<unsigned int*>(base + 2840ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2844ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2848ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2852ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2856ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2860ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2864ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2868ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2872ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2876ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2880ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 2884ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2888ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2892ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2896ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2900ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2904ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2908ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 2912ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 2916ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 2920ull * cap)[idx] = tid;
            return;
        case 27: // traverse_cylinder_fin
            reinterpret_cast<unsigned int*>(base + 2928ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 2932ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 2936ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2940ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 2944ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2948ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 2952ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2956ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 2960ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 2964ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 2968ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 2972ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 2976ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 2980ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 2984ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 2988ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 2992ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 2996ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 3000ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 3004ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 3008ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 3012ull * cap)[idx] = R.r49;
            reinterpret_cast<unsigned int*>(base + 3016ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 3020ull * cap)[idx] = tid;
            return;
        case 28: // traverse_disk
            reinterpret_cast<unsigned int*>(base + 3024ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 3028ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 3032ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 3036ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 3040ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 3044ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 3048ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 3052ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 3056ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 3060ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 3064ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 3068ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 3072ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 3076ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 3080ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 3084ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 3088ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 3092ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 3096ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 3100ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 3104ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 3108ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 3112ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 3116ull * cap)[idx] = R.r33;
            reinterpret_cast<float*>(base + 3120ull * cap)[idx] = R.r34;
            reinterpret_cast<unsigned int*>(base + 3124ull * cap)[idx] = R.r35;
            reinterpret_cast<float*>(base + 3128ull * cap)[idx] = R.r36;
            reinterpret_cast<unsigned*>(base + 3132ull * cap)[idx] = tid;
            return;
        case 29: // isect_disk_rest
            reinterpret_cast<unsigned int*>(base + 3136ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 3140ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 3144ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 3148ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 3152ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 3156ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 3160ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 3164ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 3168ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 3172ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 3176ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 3180ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 3184ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 3188ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 3192ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 3196ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 3200ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 3204ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 3208ull * cap)[idx] = R.r28;
            reinterpret_cast<float*>(base + 3212ull * cap)[idx] = R.r29;
            reinterpret_cast<float*>(base + 3216ull * cap)[idx] = R.r30;
            reinterpret_cast<float*>(base + 3220ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 3224ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 3228ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 3232ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 3236ull * cap)[idx] = tid;
            return;
        case 30: // isect_disk_end
            reinterpret_cast<unsigned int*>(base + 3240ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 3244ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 3248ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 3252ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 3256ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 3260ull * cap)[idx] = R.r6;
            reinterpret_cast<unsigned int*>(base + 3264ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 3268ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 3272ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 3276ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 3280ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 3284ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 3288ull * cap)[idx] = R.r17;
            reinterpret_cast<float*>(base + 3292ull * cap)[idx] = R.r20;
            reinterpret_cast<float*>(base + 3296ull * cap)[idx] = R.r21;
            reinterpret_cast<float*>(base + 3300ull * cap)[idx] = R.r22;
            reinterpret_cast<float*>(base + 3304ull * cap)[idx] = R.r27;
            reinterpret_cast<float*>(base + 3308ull * cap)[idx] = R.r31;
            reinterpret_cast<unsigned int*>(base + 3312ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 3316ull * cap)[idx] = R.r33;
            reinterpret_cast<unsigned int*>(base + 3320ull * cap)[idx] = R.r49;
            reinterpret_cast<unsigned int*>(base + 3324ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 3328ull * cap)[idx] = tid;
            return;
        case 31: // traverse_room_end
            reinterpret_cast<unsigned int*>(base + 3336ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 3340ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 3344ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 3348ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 3352ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 3356ull * cap)[idx] = R.r8;
            reinterpret_cast<unsigned int*>(base + 3360ull * cap)[idx] = R.r9;
            reinterpret_cast<float*>(base + 3364ull * cap)[idx] = R.r12;
            reinterpret_cast<float*>(base + 3368ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 3372ull * cap)[idx] = R.r15;
            reinterpret_cast<unsigned int*>(base + 3376ull * cap)[idx] = R.r17;
            reinterpret_cast<unsigned int*>(base + 3380ull * cap)[idx] = R.r32;
            reinterpret_cast<unsigned int*>(base + 3384ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned*>(base + 3388ull * cap)[idx] = tid;
            return;
        case 32: // fin_pixel
            reinterpret_cast<unsigned int*>(base + 3392ull * cap)[idx] = R.r1;
            reinterpret_cast<float*>(base + 3396ull * cap)[idx] = R.r2;
            reinterpret_cast<float*>(base + 3400ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 3404ull * cap)[idx] = R.r4;
            reinterpret_cast<unsigned int*>(base + 3408ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned*>(base + 3412ull * cap)[idx] = tid;
            return;
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
            R.r1 = reinterpret_cast<const unsigned int*>(base + 0ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 4ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 8ull * cap)[idx];
        case 1: // roll
            R.r1 = reinterpret_cast<const unsigned int*>(base + 16ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 20ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 24ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 28ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 32ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 36ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 40ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 44ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 48ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 52ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 56ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 60ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 64ull * cap)[idx];
        case 2: // traverse_box
            R.r1 = reinterpret_cast<const unsigned int*>(base + 72ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 76ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 80ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 84ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 88ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 92ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 96ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 100ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 104ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 108ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 112ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 116ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 120ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 124ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 128ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 132ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 136ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 140ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 144ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 148ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 152ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 156ull * cap)[idx];
        case 3: // isect_quad_l1
            R.r1 = reinterpret_cast<const unsigned int*>(base + 160ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 164ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 168ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 172ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 176ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 180ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 184ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 188ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 192ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 196ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 200ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 204ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 208ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 212ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 216ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 220ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 224ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 228ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 232ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 236ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 240ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 244ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 248ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 252ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 256ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 260ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 264ull * cap)[idx];
            R.r37 = reinterpret_cast<const float*>(base + 268ull * cap)[idx];
            R.r38 = reinterpret_cast<const float*>(base + 272ull * cap)[idx];
            R.r39 = reinterpret_cast<const float*>(base + 276ull * cap)[idx];
            R.r40 = reinterpret_cast<const float*>(base + 280ull * cap)[idx];
            R.r41 = reinterpret_cast<const float*>(base + 284ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 288ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 292ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 296ull * cap)[idx];
            R.r52 = reinterpret_cast<const float*>(base + 300ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 304ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 308ull * cap)[idx];
        case 4: // isect_quad_l2
            R.r1 = reinterpret_cast<const unsigned int*>(base + 312ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 316ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 320ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 324ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 328ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 332ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 336ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 340ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 344ull * cap)[idx];
            R.r10 = reinterpret_cast<const unsigned int*>(base + 348ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 352ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 356ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 360ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 364ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 368ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 372ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 376ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 380ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 384ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 388ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 392ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 396ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 400ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 404ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 408ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 412ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 416ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 420ull * cap)[idx];
            R.r37 = reinterpret_cast<const float*>(base + 424ull * cap)[idx];
            R.r38 = reinterpret_cast<const float*>(base + 428ull * cap)[idx];
            R.r39 = reinterpret_cast<const float*>(base + 432ull * cap)[idx];
            R.r40 = reinterpret_cast<const float*>(base + 436ull * cap)[idx];
            R.r41 = reinterpret_cast<const float*>(base + 440ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 444ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 448ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 452ull * cap)[idx];
        case 5: // isect_quad_l3
            R.r1 = reinterpret_cast<const unsigned int*>(base + 456ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 460ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 464ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 468ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 472ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 476ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 480ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 484ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 488ull * cap)[idx];
            R.r10 = reinterpret_cast<const unsigned int*>(base + 492ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 496ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 500ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 504ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 508ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 512ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 516ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 520ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 524ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 528ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 532ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 536ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 540ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 544ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 548ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 552ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 556ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 560ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 564ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 568ull * cap)[idx];
            R.r37 = reinterpret_cast<const float*>(base + 572ull * cap)[idx];
            R.r38 = reinterpret_cast<const float*>(base + 576ull * cap)[idx];
            R.r39 = reinterpret_cast<const float*>(base + 580ull * cap)[idx];
            R.r40 = reinterpret_cast<const float*>(base + 584ull * cap)[idx];
            R.r41 = reinterpret_cast<const float*>(base + 588ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 592ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 596ull * cap)[idx];
        case 6: // isect_quad_l4
            R.r1 = reinterpret_cast<const unsigned int*>(base + 600ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 604ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 608ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 612ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 616ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 620ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 624ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 628ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 632ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 636ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 640ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 644ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 648ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 652ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 656ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 660ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 664ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 668ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 672ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 676ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 680ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 684ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 688ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 692ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 696ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 700ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 704ull * cap)[idx];
            R.r37 = reinterpret_cast<const float*>(base + 708ull * cap)[idx];
            R.r38 = reinterpret_cast<const float*>(base + 712ull * cap)[idx];
            R.r39 = reinterpret_cast<const float*>(base + 716ull * cap)[idx];
            R.r40 = reinterpret_cast<const float*>(base + 720ull * cap)[idx];
            R.r41 = reinterpret_cast<const float*>(base + 724ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 728ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 732ull * cap)[idx];
        case 7: // isect_quad_l5
            R.r1 = reinterpret_cast<const unsigned int*>(base + 736ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 740ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 744ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 748ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 752ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 756ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 760ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 764ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 768ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 772ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 776ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 780ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 784ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 788ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 792ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 796ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 800ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 804ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 808ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 812ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 816ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 820ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 824ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 828ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 832ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 836ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 840ull * cap)[idx];
            R.r37 = reinterpret_cast<const float*>(base + 844ull * cap)[idx];
            R.r38 = reinterpret_cast<const float*>(base + 848ull * cap)[idx];
            R.r39 = reinterpret_cast<const float*>(base + 852ull * cap)[idx];
            R.r40 = reinterpret_cast<const float*>(base + 856ull * cap)[idx];
            R.r41 = reinterpret_cast<const float*>(base + 860ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 864ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 868ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 872ull * cap)[idx];
            R.r45 = reinterpret_cast<const float*>(base + 876ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 880ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 884ull * cap)[idx];
            R.r52 = reinterpret_cast<const float*>(base + 888ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 892ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 896ull * cap)[idx];
        case 8: // isect_quad_l6
            R.r1 = reinterpret_cast<const unsigned int*>(base + 904ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 908ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 912ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 916ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 920ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 924ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 928ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 932ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 936ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 940ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 944ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 948ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 952ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 956ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 960ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 964ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 968ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 972ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 976ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 980ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 984ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 988ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 992ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 996ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 1000ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 1004ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 1008ull * cap)[idx];
            R.r40 = reinterpret_cast<const float*>(base + 1012ull * cap)[idx];
            R.r41 = reinterpret_cast<const float*>(base + 1016ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 1020ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 1024ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 1028ull * cap)[idx];
            R.r45 = reinterpret_cast<const float*>(base + 1032ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 1036ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 1040ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 1044ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 1048ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1052ull * cap)[idx];
        case 9: // isect_quad_l7
            R.r1 = reinterpret_cast<const unsigned int*>(base + 1056ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 1060ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 1064ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1068ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 1072ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 1076ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 1080ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 1084ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 1088ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 1092ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 1096ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 1100ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 1104ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 1108ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 1112ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 1116ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 1120ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 1124ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 1128ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 1132ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 1136ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 1140ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 1144ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 1148ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 1152ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 1156ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 1160ull * cap)[idx];
            R.r40 = reinterpret_cast<const float*>(base + 1164ull * cap)[idx];
            R.r41 = reinterpret_cast<const float*>(base + 1168ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 1172ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1176ull * cap)[idx];
        case 10: // isect_quad_end
            R.r1 = reinterpret_cast<const unsigned int*>(base + 1184ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 1188ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 1192ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1196ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 1200ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 1204ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 1208ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 1212ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 1216ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 1220ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 1224ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 1228ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 1232ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 1236ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 1240ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 1244ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 1248ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 1252ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 1256ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 1260ull * cap)[idx];
            R.r49 = reinterpret_cast<const unsigned int*>(base + 1264ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 1268ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1272ull * cap)[idx];
        case 11: // traverse_tetrahedron
            R.r1 = reinterpret_cast<const unsigned int*>(base + 1280ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 1284ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 1288ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1292ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 1296ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 1300ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 1304ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 1308ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 1312ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 1316ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 1320ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 1324ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 1328ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 1332ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 1336ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 1340ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 1344ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 1348ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 1352ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 1356ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1360ull * cap)[idx];
        case 12: // isect_triangle_mid1
            R.r1 = reinterpret_cast<const unsigned int*>(base + 1368ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 1372ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 1376ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1380ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 1384ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 1388ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 1392ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 1396ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 1400ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 1404ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 1408ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 1412ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 1416ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 1420ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 1424ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 1428ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 1432ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 1436ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 1440ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 1444ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 1448ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 1452ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 1456ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 1460ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 1464ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 1468ull * cap)[idx];
            R.r37 = reinterpret_cast<const float*>(base + 1472ull * cap)[idx];
            R.r38 = reinterpret_cast<const float*>(base + 1476ull * cap)[idx];
            R.r39 = reinterpret_cast<const float*>(base + 1480ull * cap)[idx];
            R.r40 = reinterpret_cast<const float*>(base + 1484ull * cap)[idx];
            R.r41 = reinterpret_cast<const float*>(base + 1488ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 1492ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 1496ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1500ull * cap)[idx];
        case 13: // isect_triangle_mid2
            R.r1 = reinterpret_cast<const unsigned int*>(base + 1504ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 1508ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 1512ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1516ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 1520ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 1524ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 1528ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 1532ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 1536ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 1540ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 1544ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 1548ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 1552ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 1556ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 1560ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 1564ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 1568ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 1572ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 1576ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 1580ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 1584ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 1588ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 1592ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 1596ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 1600ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 1604ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 1608ull * cap)[idx];
            R.r37 = reinterpret_cast<const float*>(base + 1612ull * cap)[idx];
            R.r38 = reinterpret_cast<const float*>(base + 1616ull * cap)[idx];
            R.r39 = reinterpret_cast<const float*>(base + 1620ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 1624ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1628ull * cap)[idx];
        case 14: // isect_triangle_mid3
            R.r1 = reinterpret_cast<const unsigned int*>(base + 1632ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 1636ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 1640ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1644ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 1648ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 1652ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 1656ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 1660ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 1664ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 1668ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 1672ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 1676ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 1680ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 1684ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 1688ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 1692ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 1696ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 1700ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 1704ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 1708ull * cap)[idx];
            R.r37 = reinterpret_cast<const float*>(base + 1712ull * cap)[idx];
            R.r38 = reinterpret_cast<const float*>(base + 1716ull * cap)[idx];
            R.r39 = reinterpret_cast<const float*>(base + 1720ull * cap)[idx];
            R.r40 = reinterpret_cast<const float*>(base + 1724ull * cap)[idx];
            R.r41 = reinterpret_cast<const float*>(base + 1728ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 1732ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 1736ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1740ull * cap)[idx];
        case 15: // isect_triangle_end
            R.r1 = reinterpret_cast<const unsigned int*>(base + 1744ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 1748ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 1752ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1756ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 1760ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 1764ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 1768ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 1772ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 1776ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 1780ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 1784ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 1788ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 1792ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 1796ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 1800ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 1804ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 1808ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 1812ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 1816ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 1820ull * cap)[idx];
            R.r49 = reinterpret_cast<const unsigned int*>(base + 1824ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 1828ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1832ull * cap)[idx];
        case 16: // traverse_sphere
            R.r1 = reinterpret_cast<const unsigned int*>(base + 1840ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 1844ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 1848ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1852ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 1856ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 1860ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 1864ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 1868ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 1872ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 1876ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 1880ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 1884ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 1888ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 1892ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 1896ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 1900ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 1904ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 1908ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 1912ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 1916ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1920ull * cap)[idx];
        case 17: // traverse_solve_quadratic
            R.r1 = reinterpret_cast<const unsigned int*>(base + 1928ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 1932ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 1936ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1940ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 1944ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 1948ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 1952ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 1956ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 1960ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 1964ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 1968ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 1972ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 1976ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 1980ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 1984ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 1988ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 1992ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 1996ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2000ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2004ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 2008ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 2012ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 2016ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 2020ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 2024ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2028ull * cap)[idx];
        case 18: // sq_head1
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2032ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2036ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2040ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2044ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2048ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2052ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2056ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2060ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2064ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2068ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2072ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2076ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2080ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2084ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2088ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2092ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2096ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 2100ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2104ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2108ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 2112ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 2116ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 2120ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 2124ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2128ull * cap)[idx];
        case 19: // sq_head2
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2136ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2140ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2144ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2148ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2152ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2156ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2160ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2164ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2168ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2172ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2176ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2180ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2184ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2188ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2192ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2196ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2200ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 2204ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2208ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2212ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 2216ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 2220ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 2224ull * cap)[idx];
            R.r49 = reinterpret_cast<const unsigned int*>(base + 2228ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2232ull * cap)[idx];
        case 20: // sq_mid1
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2240ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2244ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2248ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2252ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2256ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2260ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2264ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2268ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2272ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2276ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2280ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2284ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2288ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2292ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2296ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2300ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2304ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 2308ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2312ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2316ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 2320ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 2324ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 2328ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 2332ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 2336ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2340ull * cap)[idx];
        case 21: // sq_mid2
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2344ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2348ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2352ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2356ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2360ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2364ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2368ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2372ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2376ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2380ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2384ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 2388ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2392ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2396ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2400ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2404ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2408ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2412ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 2416ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2420ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2424ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 2428ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 2432ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 2436ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 2440ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2444ull * cap)[idx];
        case 22: // sq_mid
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2448ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2452ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2456ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2460ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2464ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2468ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2472ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2476ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2480ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2484ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2488ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 2492ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2496ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2500ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2504ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2508ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2512ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2516ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 2520ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2524ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2528ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 2532ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 2536ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 2540ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2544ull * cap)[idx];
        case 23: // sq_tail
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2552ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2556ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2560ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2564ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2568ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2572ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2576ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2580ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2584ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2588ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2592ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 2596ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2600ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2604ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2608ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2612ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2616ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2620ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 2624ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2628ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2632ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 2636ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 2640ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2644ull * cap)[idx];
        case 24: // sq_end
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2648ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2652ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2656ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2660ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2664ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2668ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2672ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2676ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2680ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2684ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2688ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2692ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2696ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2700ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2704ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2708ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2712ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 2716ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2720ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2724ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 2728ull * cap)[idx];
            R.r49 = reinterpret_cast<const unsigned int*>(base + 2732ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 2736ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2740ull * cap)[idx];
        case 25: // traverse_sphere_fin
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2744ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2748ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2752ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2756ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2760ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2764ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2768ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2772ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2776ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2780ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2784ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2788ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2792ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2796ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2800ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2804ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2808ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2812ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2816ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 2820ull * cap)[idx];
            R.r49 = reinterpret_cast<const unsigned int*>(base + 2824ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 2828ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2832ull * cap)[idx];
        case 26: // traverse_cylinder
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2840ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2844ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2848ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2852ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2856ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2860ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2864ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2868ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2872ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2876ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2880ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2884ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2888ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2892ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2896ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2900ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2904ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 2908ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 2912ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 2916ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2920ull * cap)[idx];
        case 27: // traverse_cylinder_fin
            R.r1 = reinterpret_cast<const unsigned int*>(base + 2928ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 2932ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 2936ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2940ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 2944ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 2948ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2952ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 2956ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2960ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 2964ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 2968ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2972ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 2976ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 2980ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 2984ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 2988ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 2992ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 2996ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 3000ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 3004ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 3008ull * cap)[idx];
            R.r49 = reinterpret_cast<const unsigned int*>(base + 3012ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 3016ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 3020ull * cap)[idx];
        case 28: // traverse_disk
            R.r1 = reinterpret_cast<const unsigned int*>(base + 3024ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 3028ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 3032ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 3036ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 3040ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 3044ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 3048ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 3052ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 3056ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 3060ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 3064ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 3068ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 3072ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 3076ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 3080ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 3084ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 3088ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 3092ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 3096ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 3100ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 3104ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 3108ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 3112ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 3116ull * cap)[idx];
            R.r34 = reinterpret_cast<const float*>(base + 3120ull * cap)[idx];
            R.r35 = reinterpret_cast<const unsigned int*>(base + 3124ull * cap)[idx];
            R.r36 = reinterpret_cast<const float*>(base + 3128ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 3132ull * cap)[idx];
        case 29: // isect_disk_rest
            R.r1 = reinterpret_cast<const unsigned int*>(base + 3136ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 3140ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 3144ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 3148ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 3152ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 3156ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 3160ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 3164ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 3168ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 3172ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 3176ull * cap)[idx];
            R.r14 = reinterpret_cast<const unsigned int*>(base + 3180ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 3184ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 3188ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 3192ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 3196ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 3200ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 3204ull * cap)[idx];
            R.r28 = reinterpret_cast<const float*>(base + 3208ull * cap)[idx];
            R.r29 = reinterpret_cast<const float*>(base + 3212ull * cap)[idx];
            R.r30 = reinterpret_cast<const float*>(base + 3216ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 3220ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 3224ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 3228ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 3232ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 3236ull * cap)[idx];
        case 30: // isect_disk_end
            R.r1 = reinterpret_cast<const unsigned int*>(base + 3240ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 3244ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 3248ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 3252ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 3256ull * cap)[idx];
            R.r6 = reinterpret_cast<const unsigned int*>(base + 3260ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 3264ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 3268ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 3272ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 3276ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 3280ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 3284ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 3288ull * cap)[idx];
            R.r20 = reinterpret_cast<const float*>(base + 3292ull * cap)[idx];
            R.r21 = reinterpret_cast<const float*>(base + 3296ull * cap)[idx];
            R.r22 = reinterpret_cast<const float*>(base + 3300ull * cap)[idx];
            R.r27 = reinterpret_cast<const float*>(base + 3304ull * cap)[idx];
            R.r31 = reinterpret_cast<const float*>(base + 3308ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 3312ull * cap)[idx];
            R.r33 = reinterpret_cast<const unsigned int*>(base + 3316ull * cap)[idx];
            R.r49 = reinterpret_cast<const unsigned int*>(base + 3320ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 3324ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 3328ull * cap)[idx];
        case 31: // traverse_room_end
            R.r1 = reinterpret_cast<const unsigned int*>(base + 3336ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 3340ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 3344ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 3348ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 3352ull * cap)[idx];
            R.r8 = reinterpret_cast<const unsigned int*>(base + 3356ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 3360ull * cap)[idx];
            R.r12 = reinterpret_cast<const float*>(base + 3364ull * cap)[idx];
            R.r13 = reinterpret_cast<const float*>(base + 3368ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 3372ull * cap)[idx];
            R.r17 = reinterpret_cast<const unsigned int*>(base + 3376ull * cap)[idx];
            R.r32 = reinterpret_cast<const unsigned int*>(base + 3380ull * cap)[idx];
            R.r53 = reinterpret_cast<const unsigned int*>(base + 3384ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 3388ull * cap)[idx];
        case 32: // fin_pixel
            R.r1 = reinterpret_cast<const unsigned int*>(base + 3392ull * cap)[idx];
            R.r2 = reinterpret_cast<const float*>(base + 3396ull * cap)[idx];
            R.r3 = reinterpret_cast<const float*>(base + 3400ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 3404ull * cap)[idx];
            R.r5 = reinterpret_cast<const unsigned int*>(base + 3408ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 3412ull * cap)[idx];
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
const unsigned long long kQOffs0[] = {0ull, 4ull};
const uint32_t kQRegs1[] = {1u, 2u, 3u, 4u, 5u, 8u, 9u, 12u, 13u, 15u, 17u, 53u};
const int kQTypes1[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames1[] = {"ppp", "L0", "L1", "L2", "rc", "c0", "c1", "pp0", "pp1", "pw", "sc", "ct"};
const unsigned long long kQOffs1[] = {16ull, 20ull, 24ull, 28ull, 32ull, 36ull, 40ull, 44ull, 48ull, 52ull, 56ull, 60ull};
const uint32_t kQRegs2[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 53u};
const int kQTypes2[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames2[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "ct"};
const unsigned long long kQOffs2[] = {72ull, 76ull, 80ull, 84ull, 88ull, 92ull, 96ull, 100ull, 104ull, 108ull, 112ull, 116ull, 120ull, 124ull, 128ull, 132ull, 136ull, 140ull, 144ull, 148ull, 152ull};
const uint32_t kQRegs3[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 50u, 51u, 52u, 53u};
const int kQTypes3[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames3[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "vr60", "vr61", "vr62", "ct"};
const unsigned long long kQOffs3[] = {160ull, 164ull, 168ull, 172ull, 176ull, 180ull, 184ull, 188ull, 192ull, 196ull, 200ull, 204ull, 208ull, 212ull, 216ull, 220ull, 224ull, 228ull, 232ull, 236ull, 240ull, 244ull, 248ull, 252ull, 256ull, 260ull, 264ull, 268ull, 272ull, 276ull, 280ull, 284ull, 288ull, 292ull, 296ull, 300ull, 304ull};
const uint32_t kQRegs4[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 10u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 53u};
const int kQTypes4[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames4[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "tmp1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct"};
const unsigned long long kQOffs4[] = {312ull, 316ull, 320ull, 324ull, 328ull, 332ull, 336ull, 340ull, 344ull, 348ull, 352ull, 356ull, 360ull, 364ull, 368ull, 372ull, 376ull, 380ull, 384ull, 388ull, 392ull, 396ull, 400ull, 404ull, 408ull, 412ull, 416ull, 420ull, 424ull, 428ull, 432ull, 436ull, 440ull, 444ull, 448ull};
const uint32_t kQRegs5[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 10u, 11u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u};
const int kQTypes5[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames5[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "tmp1", "tmp2", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32"};
const unsigned long long kQOffs5[] = {456ull, 460ull, 464ull, 468ull, 472ull, 476ull, 480ull, 484ull, 488ull, 492ull, 496ull, 500ull, 504ull, 508ull, 512ull, 516ull, 520ull, 524ull, 528ull, 532ull, 536ull, 540ull, 544ull, 548ull, 552ull, 556ull, 560ull, 564ull, 568ull, 572ull, 576ull, 580ull, 584ull, 588ull, 592ull};
const uint32_t kQRegs6[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u};
const int kQTypes6[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames6[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32"};
const unsigned long long kQOffs6[] = {600ull, 604ull, 608ull, 612ull, 616ull, 620ull, 624ull, 628ull, 632ull, 636ull, 640ull, 644ull, 648ull, 652ull, 656ull, 660ull, 664ull, 668ull, 672ull, 676ull, 680ull, 684ull, 688ull, 692ull, 696ull, 700ull, 704ull, 708ull, 712ull, 716ull, 720ull, 724ull, 728ull};
const uint32_t kQRegs7[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 43u, 44u, 45u, 50u, 51u, 52u, 53u};
const int kQTypes7[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames7[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "vr40", "vr41", "vr42", "vr60", "vr61", "vr62", "ct"};
const unsigned long long kQOffs7[] = {736ull, 740ull, 744ull, 748ull, 752ull, 756ull, 760ull, 764ull, 768ull, 772ull, 776ull, 780ull, 784ull, 788ull, 792ull, 796ull, 800ull, 804ull, 808ull, 812ull, 816ull, 820ull, 824ull, 828ull, 832ull, 836ull, 840ull, 844ull, 848ull, 852ull, 856ull, 860ull, 864ull, 868ull, 872ull, 876ull, 880ull, 884ull, 888ull, 892ull};
const uint32_t kQRegs8[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 40u, 41u, 42u, 43u, 44u, 45u, 46u, 47u, 48u, 53u};
const int kQTypes8[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames8[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr30", "vr31", "vr32", "vr40", "vr41", "vr42", "vr50", "vr51", "vr52", "ct"};
const unsigned long long kQOffs8[] = {904ull, 908ull, 912ull, 916ull, 920ull, 924ull, 928ull, 932ull, 936ull, 940ull, 944ull, 948ull, 952ull, 956ull, 960ull, 964ull, 968ull, 972ull, 976ull, 980ull, 984ull, 988ull, 992ull, 996ull, 1000ull, 1004ull, 1008ull, 1012ull, 1016ull, 1020ull, 1024ull, 1028ull, 1032ull, 1036ull, 1040ull, 1044ull, 1048ull};
const uint32_t kQRegs9[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 40u, 41u, 42u};
const int kQTypes9[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames9[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr30", "vr31", "vr32"};
const unsigned long long kQOffs9[] = {1056ull, 1060ull, 1064ull, 1068ull, 1072ull, 1076ull, 1080ull, 1084ull, 1088ull, 1092ull, 1096ull, 1100ull, 1104ull, 1108ull, 1112ull, 1116ull, 1120ull, 1124ull, 1128ull, 1132ull, 1136ull, 1140ull, 1144ull, 1148ull, 1152ull, 1156ull, 1160ull, 1164ull, 1168ull, 1172ull};
const uint32_t kQRegs10[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes10[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames10[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs10[] = {1184ull, 1188ull, 1192ull, 1196ull, 1200ull, 1204ull, 1208ull, 1212ull, 1216ull, 1220ull, 1224ull, 1228ull, 1232ull, 1236ull, 1240ull, 1244ull, 1248ull, 1252ull, 1256ull, 1260ull, 1264ull, 1268ull};
const uint32_t kQRegs11[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u};
const int kQTypes11[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames11[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp"};
const unsigned long long kQOffs11[] = {1280ull, 1284ull, 1288ull, 1292ull, 1296ull, 1300ull, 1304ull, 1308ull, 1312ull, 1316ull, 1320ull, 1324ull, 1328ull, 1332ull, 1336ull, 1340ull, 1344ull, 1348ull, 1352ull, 1356ull};
const uint32_t kQRegs12[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 40u, 41u, 42u, 53u};
const int kQTypes12[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames12[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct"};
const unsigned long long kQOffs12[] = {1368ull, 1372ull, 1376ull, 1380ull, 1384ull, 1388ull, 1392ull, 1396ull, 1400ull, 1404ull, 1408ull, 1412ull, 1416ull, 1420ull, 1424ull, 1428ull, 1432ull, 1436ull, 1440ull, 1444ull, 1448ull, 1452ull, 1456ull, 1460ull, 1464ull, 1468ull, 1472ull, 1476ull, 1480ull, 1484ull, 1488ull, 1492ull, 1496ull};
const uint32_t kQRegs13[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u, 37u, 38u, 39u, 53u};
const int kQTypes13[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames13[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12", "vr20", "vr21", "vr22", "ct"};
const unsigned long long kQOffs13[] = {1504ull, 1508ull, 1512ull, 1516ull, 1520ull, 1524ull, 1528ull, 1532ull, 1536ull, 1540ull, 1544ull, 1548ull, 1552ull, 1556ull, 1560ull, 1564ull, 1568ull, 1572ull, 1576ull, 1580ull, 1584ull, 1588ull, 1592ull, 1596ull, 1600ull, 1604ull, 1608ull, 1612ull, 1616ull, 1620ull, 1624ull};
const uint32_t kQRegs14[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 37u, 38u, 39u, 40u, 41u, 42u, 53u};
const int kQTypes14[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames14[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "vr20", "vr21", "vr22", "vr30", "vr31", "vr32", "ct"};
const unsigned long long kQOffs14[] = {1632ull, 1636ull, 1640ull, 1644ull, 1648ull, 1652ull, 1656ull, 1660ull, 1664ull, 1668ull, 1672ull, 1676ull, 1680ull, 1684ull, 1688ull, 1692ull, 1696ull, 1700ull, 1704ull, 1708ull, 1712ull, 1716ull, 1720ull, 1724ull, 1728ull, 1732ull, 1736ull};
const uint32_t kQRegs15[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes15[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames15[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs15[] = {1744ull, 1748ull, 1752ull, 1756ull, 1760ull, 1764ull, 1768ull, 1772ull, 1776ull, 1780ull, 1784ull, 1788ull, 1792ull, 1796ull, 1800ull, 1804ull, 1808ull, 1812ull, 1816ull, 1820ull, 1824ull, 1828ull};
const uint32_t kQRegs16[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 53u};
const int kQTypes16[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames16[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "ct"};
const unsigned long long kQOffs16[] = {1840ull, 1844ull, 1848ull, 1852ull, 1856ull, 1860ull, 1864ull, 1868ull, 1872ull, 1876ull, 1880ull, 1884ull, 1888ull, 1892ull, 1896ull, 1900ull, 1904ull, 1908ull, 1912ull, 1916ull};
const uint32_t kQRegs17[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 34u, 35u, 36u, 53u};
const int kQTypes17[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames17[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "ct"};
const unsigned long long kQOffs17[] = {1928ull, 1932ull, 1936ull, 1940ull, 1944ull, 1948ull, 1952ull, 1956ull, 1960ull, 1964ull, 1968ull, 1972ull, 1976ull, 1980ull, 1984ull, 1988ull, 1992ull, 1996ull, 2000ull, 2004ull, 2008ull, 2012ull, 2016ull, 2020ull, 2024ull};
const uint32_t kQRegs18[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 35u, 36u, 53u};
const int kQTypes18[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames18[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr11", "vr12", "ct"};
const unsigned long long kQOffs18[] = {2032ull, 2036ull, 2040ull, 2044ull, 2048ull, 2052ull, 2056ull, 2060ull, 2064ull, 2068ull, 2072ull, 2076ull, 2080ull, 2084ull, 2088ull, 2092ull, 2096ull, 2100ull, 2104ull, 2108ull, 2112ull, 2116ull, 2120ull, 2124ull};
const uint32_t kQRegs19[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 35u, 36u, 49u};
const int kQTypes19[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames19[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr11", "vr12", "hit"};
const unsigned long long kQOffs19[] = {2136ull, 2140ull, 2144ull, 2148ull, 2152ull, 2156ull, 2160ull, 2164ull, 2168ull, 2172ull, 2176ull, 2180ull, 2184ull, 2188ull, 2192ull, 2196ull, 2200ull, 2204ull, 2208ull, 2212ull, 2216ull, 2220ull, 2224ull, 2228ull};
const uint32_t kQRegs20[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 34u, 35u, 36u, 53u};
const int kQTypes20[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames20[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12", "ct"};
const unsigned long long kQOffs20[] = {2240ull, 2244ull, 2248ull, 2252ull, 2256ull, 2260ull, 2264ull, 2268ull, 2272ull, 2276ull, 2280ull, 2284ull, 2288ull, 2292ull, 2296ull, 2300ull, 2304ull, 2308ull, 2312ull, 2316ull, 2320ull, 2324ull, 2328ull, 2332ull, 2336ull};
const uint32_t kQRegs21[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 34u, 35u, 36u};
const int kQTypes21[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32};
const char* const kQNames21[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr10", "vr11", "vr12"};
const unsigned long long kQOffs21[] = {2344ull, 2348ull, 2352ull, 2356ull, 2360ull, 2364ull, 2368ull, 2372ull, 2376ull, 2380ull, 2384ull, 2388ull, 2392ull, 2396ull, 2400ull, 2404ull, 2408ull, 2412ull, 2416ull, 2420ull, 2424ull, 2428ull, 2432ull, 2436ull, 2440ull};
const uint32_t kQRegs22[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 36u, 53u};
const int kQTypes22[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames22[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "vr12", "ct"};
const unsigned long long kQOffs22[] = {2448ull, 2452ull, 2456ull, 2460ull, 2464ull, 2468ull, 2472ull, 2476ull, 2480ull, 2484ull, 2488ull, 2492ull, 2496ull, 2500ull, 2504ull, 2508ull, 2512ull, 2516ull, 2520ull, 2524ull, 2528ull, 2532ull, 2536ull, 2540ull};
const uint32_t kQRegs23[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 53u};
const int kQTypes23[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames23[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "ct"};
const unsigned long long kQOffs23[] = {2552ull, 2556ull, 2560ull, 2564ull, 2568ull, 2572ull, 2576ull, 2580ull, 2584ull, 2588ull, 2592ull, 2596ull, 2600ull, 2604ull, 2608ull, 2612ull, 2616ull, 2620ull, 2624ull, 2628ull, 2632ull, 2636ull, 2640ull};
const uint32_t kQRegs24[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes24[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames24[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs24[] = {2648ull, 2652ull, 2656ull, 2660ull, 2664ull, 2668ull, 2672ull, 2676ull, 2680ull, 2684ull, 2688ull, 2692ull, 2696ull, 2700ull, 2704ull, 2708ull, 2712ull, 2716ull, 2720ull, 2724ull, 2728ull, 2732ull, 2736ull};
const uint32_t kQRegs25[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes25[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames25[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs25[] = {2744ull, 2748ull, 2752ull, 2756ull, 2760ull, 2764ull, 2768ull, 2772ull, 2776ull, 2780ull, 2784ull, 2788ull, 2792ull, 2796ull, 2800ull, 2804ull, 2808ull, 2812ull, 2816ull, 2820ull, 2824ull, 2828ull};
const uint32_t kQRegs26[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 53u};
const int kQTypes26[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames26[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "ct"};
const unsigned long long kQOffs26[] = {2840ull, 2844ull, 2848ull, 2852ull, 2856ull, 2860ull, 2864ull, 2868ull, 2872ull, 2876ull, 2880ull, 2884ull, 2888ull, 2892ull, 2896ull, 2900ull, 2904ull, 2908ull, 2912ull, 2916ull};
const uint32_t kQRegs27[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 29u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes27[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames27[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "vr01", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs27[] = {2928ull, 2932ull, 2936ull, 2940ull, 2944ull, 2948ull, 2952ull, 2956ull, 2960ull, 2964ull, 2968ull, 2972ull, 2976ull, 2980ull, 2984ull, 2988ull, 2992ull, 2996ull, 3000ull, 3004ull, 3008ull, 3012ull, 3016ull};
const uint32_t kQRegs28[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 34u, 35u, 36u};
const int kQTypes28[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32};
const char* const kQNames28[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "vr10", "vr11", "vr12"};
const unsigned long long kQOffs28[] = {3024ull, 3028ull, 3032ull, 3036ull, 3040ull, 3044ull, 3048ull, 3052ull, 3056ull, 3060ull, 3064ull, 3068ull, 3072ull, 3076ull, 3080ull, 3084ull, 3088ull, 3092ull, 3096ull, 3100ull, 3104ull, 3108ull, 3112ull, 3116ull, 3120ull, 3124ull, 3128ull};
const uint32_t kQRegs29[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 14u, 15u, 17u, 20u, 21u, 22u, 27u, 28u, 29u, 30u, 31u, 32u, 33u, 53u};
const int kQTypes29[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames29[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "tmp0", "pw", "sc", "o0", "o1", "o2", "d2", "vr00", "vr01", "vr02", "t", "pid", "rp", "ct"};
const unsigned long long kQOffs29[] = {3136ull, 3140ull, 3144ull, 3148ull, 3152ull, 3156ull, 3160ull, 3164ull, 3168ull, 3172ull, 3176ull, 3180ull, 3184ull, 3188ull, 3192ull, 3196ull, 3200ull, 3204ull, 3208ull, 3212ull, 3216ull, 3220ull, 3224ull, 3228ull, 3232ull};
const uint32_t kQRegs30[] = {1u, 2u, 3u, 4u, 5u, 6u, 7u, 8u, 9u, 12u, 13u, 15u, 17u, 20u, 21u, 22u, 27u, 31u, 32u, 33u, 49u, 53u};
const int kQTypes30[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames30[] = {"ppp", "L0", "L1", "L2", "rc", "d0", "d1", "c0", "c1", "pp0", "pp1", "pw", "sc", "o0", "o1", "o2", "d2", "t", "pid", "rp", "hit", "ct"};
const unsigned long long kQOffs30[] = {3240ull, 3244ull, 3248ull, 3252ull, 3256ull, 3260ull, 3264ull, 3268ull, 3272ull, 3276ull, 3280ull, 3284ull, 3288ull, 3292ull, 3296ull, 3300ull, 3304ull, 3308ull, 3312ull, 3316ull, 3320ull, 3324ull};
const uint32_t kQRegs31[] = {1u, 2u, 3u, 4u, 5u, 8u, 9u, 12u, 13u, 15u, 17u, 32u, 53u};
const int kQTypes31[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames31[] = {"ppp", "L0", "L1", "L2", "rc", "c0", "c1", "pp0", "pp1", "pw", "sc", "pid", "ct"};
const unsigned long long kQOffs31[] = {3336ull, 3340ull, 3344ull, 3348ull, 3352ull, 3356ull, 3360ull, 3364ull, 3368ull, 3372ull, 3376ull, 3380ull, 3384ull};
const uint32_t kQRegs32[] = {1u, 2u, 3u, 4u, 5u};
const int kQTypes32[] = {LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames32[] = {"ppp", "L0", "L1", "L2", "rc"};
const unsigned long long kQOffs32[] = {3392ull, 3396ull, 3400ull, 3404ull, 3408ull};
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
    {kQOffs0, 8ull},
    {kQOffs1, 64ull},
    {kQOffs2, 156ull},
    {kQOffs3, 308ull},
    {kQOffs4, 452ull},
    {kQOffs5, 596ull},
    {kQOffs6, 732ull},
    {kQOffs7, 896ull},
    {kQOffs8, 1052ull},
    {kQOffs9, 1176ull},
    {kQOffs10, 1272ull},
    {kQOffs11, 1360ull},
    {kQOffs12, 1500ull},
    {kQOffs13, 1628ull},
    {kQOffs14, 1740ull},
    {kQOffs15, 1832ull},
    {kQOffs16, 1920ull},
    {kQOffs17, 2028ull},
    {kQOffs18, 2128ull},
    {kQOffs19, 2232ull},
    {kQOffs20, 2340ull},
    {kQOffs21, 2444ull},
    {kQOffs22, 2544ull},
    {kQOffs23, 2644ull},
    {kQOffs24, 2740ull},
    {kQOffs25, 2832ull},
    {kQOffs26, 2920ull},
    {kQOffs27, 3020ull},
    {kQOffs28, 3132ull},
    {kQOffs29, 3236ull},
    {kQOffs30, 3328ull},
    {kQOffs31, 3388ull},
    {kQOffs32, 3412ull},
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

/// The megakernel at register cap `regs` (0: the default); profiled
/// launches use the default cap.  NULL: no such cap compiled.
const void* regroup_fn(unsigned regs, bool profile)
{
    if(profile) return reinterpret_cast<const void*>(&regroup_kernel<K, true, K::kRegroupMaxRegs>);
    switch(regs)
    {
    case 0u:
    case 64u: return reinterpret_cast<const void*>(&regroup_kernel<K, false, 64>);
    case 32u: return reinterpret_cast<const void*>(&regroup_kernel<K, false, 32>);
    case 40u: return reinterpret_cast<const void*>(&regroup_kernel<K, false, 40>);
    case 48u: return reinterpret_cast<const void*>(&regroup_kernel<K, false, 48>);
    case 56u: return reinterpret_cast<const void*>(&regroup_kernel<K, false, 56>);
    case 80u: return reinterpret_cast<const void*>(&regroup_kernel<K, false, 80>);
    case 96u: return reinterpret_cast<const void*>(&regroup_kernel<K, false, 96>);
    case 128u: return reinterpret_cast<const void*>(&regroup_kernel<K, false, 128>);
    default: return nullptr;
    }
}

cudaError_t launch_regroup(const RegroupLaunch& a)
{
    void* args[] = {const_cast<RegroupParams*>(&a.params)};
    const void* fn = regroup_fn(a.regs, a.profile);
    if(!fn) return cudaErrorInvalidValue;
    if(a.ordinary && a.params.slice_rounds == 1u)
        return cudaLaunchKernel(fn, dim3(a.grid), dim3(a.block), args, 0, a.stream);
    return cudaLaunchCooperativeKernel(fn, dim3(a.grid), dim3(a.block), args, 0, a.stream);
}

cudaError_t regroup_occupancy(int block, bool profile, unsigned regs, int* ctas)
{
    const void* fn = regroup_fn(regs, profile);
    if(!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, 0);
}

} } // namespace loom_b200::k_primary_const_b20_256

extern const loom_b200::KernelEntry loom_b200_entry_primary_const_b20_256;
const loom_b200::KernelEntry loom_b200_entry_primary_const_b20_256 = {
    &loom_b200::k_primary_const_b20_256::kInfo, loom_b200::k_primary_const_b20_256::K::kRowBytes, 33,
    &loom_b200::k_primary_const_b20_256::launch_plain, &loom_b200::k_primary_const_b20_256::launch_regroup,
    &loom_b200::k_primary_const_b20_256::regroup_occupancy,
    loom_b200::k_primary_const_b20_256::kQueues, loom_b200::k_primary_const_b20_256::kSegments,
    loom_b200::k_primary_const_b20_256::kRegCaps, 8u};
