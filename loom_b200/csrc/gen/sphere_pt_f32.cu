// Generated by loom_b200.codegen from loom_b200/ir/sphere_pt_f32.lir.
// Kernel IR digest 144eab9a4253b9da; regenerate instead of editing.
#include "../engine/plain.cuh"
#include "../engine/regroup.cuh"
#include "../runtime_iface.h"

namespace loom_b200 { namespace k_sphere_pt_f32 {

__constant__ unsigned kInstrTab[24] = {32, 63, 5, 38, 2, 28, 4, 3, 2, 2, 4, 4, 18, 5, 26, 2, 8, 20, 13, 40, 2, 4, 7, 292};
__constant__ unsigned kLiveTab[28] = {8, 68, 76, 92, 84, 84, 36, 104, 104, 104, 108, 108, 104, 92, 76, 100, 108, 112, 108, 108, 120, 96, 80, 220, 60, 104, 100, 116};
__constant__ int kQueueBlock[28] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 23, 23, 23, 23};
__constant__ unsigned kQuorumTab[24] = {27, 18, 0, 8, 0, 4, 0, 0, 0, 0, 0, 0, 0, 0, 5, 0, 0, 0, 0, 6, 0, 0, 0, 22};
__constant__ unsigned kRankTab[24] = {0, 9, 10, 11, 12, 13, 14, 15, 16, 17, 7, 8, 18, 21, 22, 23, 5, 6, 19, 20, 2, 3, 4, 1};

struct K
{
    static constexpr int kNumBlocks = 24;
    static constexpr int kNumQueues = 28;
    static constexpr int kRegroupMaxRegs = 64;
    static constexpr bool kSplitCallSites = false;
    struct Regs
    {
        unsigned int r1; // inst: u32
        unsigned int r2; // sid: u32
        float r3; // L0: f32
        float r4; // L1: f32
        float r5; // L2: f32
        unsigned int r6; // hb: u32
        unsigned int r7; // w: u32
        unsigned int r8; // ti: u32
        unsigned int r9; // h: u32
        unsigned int r10; // sl: u32
        unsigned int r11; // k0: u32
        unsigned int r12; // soff: u32
        unsigned int r13; // scnt: u32
        float r14; // cam0: f32
        float r15; // cam1: f32
        float r16; // cam2: f32
        float r17; // tanf: f32
        unsigned int r18; // pix: u32
        unsigned int r19; // msk: u32
        unsigned int r20; // smp: u32
        unsigned int r21; // px: u32
        unsigned int r22; // py: u32
        unsigned int r23; // k2: u32
        unsigned int r24; // c0: u32
        unsigned int r25; // c1: u32
        unsigned int r26; // rpt: u32
        unsigned int r27; // sub: u32
        unsigned int r28; // sbx: u32
        unsigned int r29; // sby: u32
        float r30; // ra: f32
        float r31; // fa: f32
        float r32; // fb: f32
        unsigned int r33; // cnd: u32
        float r34; // fdx: f32
        float r35; // fdy: f32
        float r36; // fx: f32
        float r37; // fp: f32
        float r38; // fy: f32
        float r39; // fw: f32
        float r40; // fh: f32
        float r41; // asp: f32
        float r42; // d0: f32
        float r43; // d1: f32
        float r44; // d2: f32
        float r45; // tmp: f32
        float r46; // o0: f32
        float r47; // o1: f32
        float r48; // o2: f32
        float r49; // T0: f32
        float r50; // T1: f32
        float r51; // T2: f32
        unsigned int r52; // depth: u32
        float r53; // tmin: f32
        unsigned int r54; // hid: u32
        unsigned int r55; // i: u32
        unsigned int r56; // sp: u32
        float r57; // s0: f32
        float r58; // s1: f32
        float r59; // s2: f32
        float r60; // sr: f32
        float r61; // oc0: f32
        float r62; // oc1: f32
        float r63; // oc2: f32
        float r64; // bq: f32
        float r65; // nbq: f32
        float r66; // q0: f32
        float r67; // q1: f32
        float r68; // q2: f32
        float r69; // l2: f32
        float r70; // det: f32
        unsigned int r71; // hit: u32
        float r72; // sq: f32
        float r73; // t0: f32
        float r74; // t1: f32
        float r75; // tt: f32
        float r76; // cr: f32
        float r77; // cg: f32
        float r78; // cb: f32
        unsigned int r79; // mat: u32
        float r80; // x0: f32
        float r81; // x1: f32
        float r82; // x2: f32
        float r83; // n0: f32
        float r84; // n1: f32
        float r85; // n2: f32
        float r86; // p: f32
        float r87; // dn: f32
        unsigned int r88; // into: u32
        float r89; // m0: f32
        float r90; // m1: f32
        float r91; // m2: f32
        float r92; // nl0: f32
        float r93; // nl1: f32
        float r94; // nl2: f32
        float r95; // dn2: f32
        float r96; // aw: f32
        float r97; // a0: f32
        float r98; // a1: f32
        float r99; // a2: f32
        float r100; // uu0: f32
        float r101; // uu1: f32
        float r102; // uu2: f32
        float r103; // vv0: f32
        float r104; // vv1: f32
        float r105; // vv2: f32
        float r106; // dx: f32
        float r107; // dy: f32
        float r108; // rr2: f32
        float r109; // dz: f32
        float r110; // nin: f32
        float r111; // nnt: f32
        float r112; // ddn: f32
        float r113; // c2: f32
        float r114; // nn2: f32
        float r115; // sc: f32
        float r116; // nsc: f32
        float r117; // td0: f32
        float r118; // td1: f32
        float r119; // td2: f32
        float r120; // r0: f32
        float r121; // ctn: f32
        float r122; // nddn: f32
        float r123; // cc: f32
        float r124; // c5: f32
        float r125; // re: f32
        float r126; // tr: f32
        float r127; // pp: f32
        float r128; // rp: f32
        float r129; // tp: f32
        unsigned int r130; // u0: f32,u32
        unsigned int r131; // u1: f32,u32
        unsigned int r132; // tmp1: u32
        unsigned int r133; // tmp2: u32
    };

    struct In
    {
        unsigned int v0; // inst
        unsigned int v1; // sid
    };

    // Reads the input columns of thread `tid` (a NULL column is iota).
    __device__ __forceinline__ static void
    load_in(In& in, const Columns& c, const unsigned long long tid)
    {
        in.v0 = load_input<unsigned int>(c, 0, tid);
        in.v1 = load_input<unsigned int>(c, 1, tid);
        (void)in; (void)c; (void)tid;
    }

    // Loom's set_inputs: input variables written, every other register zero.
    // Only registers live at START (those its queue carries) are written:
    // the others are written before they are read on every path.
    __device__ __forceinline__ static void
    start(Regs& R, const In& in)
    {
        R.r1 = static_cast<unsigned int>(in.v0);
        R.r2 = static_cast<unsigned int>(in.v1);
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
        static_cast<float*>(c.p[2])[col_index(c, tid)] = R.r3; // L0
        static_cast<float*>(c.p[3])[col_index(c, tid)] = R.r4; // L1
        static_cast<float*>(c.p[4])[col_index(c, tid)] = R.r5; // L2
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
        case 0: return 23;
        default: return -1;
        }
    }

    static constexpr int kMaxQueuesPerBlock = 5;
    // j-th queue holding threads that stand at block b (-1: none).
    __device__ __forceinline__ static int
    queue_list(const int b, const int j)
    {
        if(b == 23)
        {
            switch(j)
            {
            case 0: return 23;
            case 1: return 24;
            case 2: return 25;
            case 3: return 26;
            case 4: return 27;
            default: return -1;
            }
        }
        return j == 0 ? b : -1;
    }

    // Queue a thread standing at block pc waits in: the block's own queue,
    // or for a dispatch block the queue of the context its register selects.
    __device__ __forceinline__ static int
    queue_of(const int pc, const Regs& R)
    {
        (void)R;
        if(pc == 23)
        {
            switch(static_cast<unsigned long long>(R.r26))
            {
            case 0ull: return 24;
            case 1ull: return 25;
            case 2ull: return 26;
            case 3ull: return 27;
            default: break;
            }
        }
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
        default: return kHalt;
        }
    L_B0: // START
        if(stop_heavy && !fresh) return 0;
    L_B0_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 0, 32u);
        R.r6 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r1) * static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r7 = static_cast<unsigned int>(table_load<unsigned int>(*ctx.cols, static_cast<unsigned>(R.r6)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r6) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r9 = static_cast<unsigned int>(table_load<unsigned int>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r6) + static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r10 = static_cast<unsigned int>(table_load<unsigned int>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r6) + static_cast<unsigned int>(((unsigned int)0x3ull))));
        R.r11 = static_cast<unsigned int>(table_load<unsigned int>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r6) + static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r12 = static_cast<unsigned int>(table_load<unsigned int>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r6) + static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r13 = static_cast<unsigned int>(table_load<unsigned int>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r6) + static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r14 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r6) + static_cast<unsigned int>(((unsigned int)0x7ull))));
        R.r15 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r6) + static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r16 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r6) + static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r17 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r18 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r2) >> static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1ull)) << static_cast<unsigned int>(R.r10)));
        R.r19 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r19) - static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r20 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r2) & static_cast<unsigned int>(R.r19)));
        R.r21 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) % static_cast<unsigned int>(R.r7)));
        R.r22 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r18) / static_cast<unsigned int>(R.r7)));
        R.r23 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r11) ^ static_cast<unsigned int>(((unsigned int)0x1bd11bdaull))));
        R.r23 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r23) ^ static_cast<unsigned int>(((unsigned int)0x9e3779b9ull))));
        R.r24 = static_cast<unsigned int>(R.r18);
        R.r25 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) << static_cast<unsigned int>(((unsigned int)0x14ull))));
        R.r26 = static_cast<unsigned int>(((unsigned int)0x0ull));
        goto L_B23;
    L_B1: // prim
        if(stop_heavy && !fresh) return 1;
    L_B1_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 1, 63u);
        R.r27 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r20) & static_cast<unsigned int>(((unsigned int)0x3ull))));
        R.r28 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r27) & static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r29 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r27) >> static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r30 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r130)) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r31 = static_cast<float>(op_sqrt(static_cast<float>(R.r30)));
        R.r31 = static_cast<float>(static_cast<float>(static_cast<float>(R.r31) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r32 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+1f)) - static_cast<float>(R.r30)));
        R.r32 = static_cast<float>(op_sqrt(static_cast<float>(R.r32)));
        R.r32 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r32)));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r30) < static_cast<float>((0x1.0000000000000p+0f))));
        R.r34 = static_cast<float>(((R.r33) ? (R.r31) : (R.r32)));
        R.r30 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r131)) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r31 = static_cast<float>(op_sqrt(static_cast<float>(R.r30)));
        R.r31 = static_cast<float>(static_cast<float>(static_cast<float>(R.r31) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r32 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+1f)) - static_cast<float>(R.r30)));
        R.r32 = static_cast<float>(op_sqrt(static_cast<float>(R.r32)));
        R.r32 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r32)));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r30) < static_cast<float>((0x1.0000000000000p+0f))));
        R.r35 = static_cast<float>(((R.r33) ? (R.r31) : (R.r32)));
        R.r36 = static_cast<float>(R.r28);
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) + static_cast<float>((0x1.0000000000000p-1f))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) + static_cast<float>(R.r34)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>((0x1.0000000000000p-1f))));
        R.r37 = static_cast<float>(R.r21);
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) + static_cast<float>(R.r37)));
        R.r38 = static_cast<float>(R.r29);
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) + static_cast<float>((0x1.0000000000000p-1f))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) + static_cast<float>(R.r35)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>((0x1.0000000000000p-1f))));
        R.r37 = static_cast<float>(R.r22);
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) + static_cast<float>(R.r37)));
        R.r39 = static_cast<float>(R.r7);
        R.r40 = static_cast<float>(R.r9);
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) / static_cast<float>(R.r39)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r41 = static_cast<float>(static_cast<float>(static_cast<float>(R.r39) / static_cast<float>(R.r40)));
        R.r36 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(R.r41)));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r36) * static_cast<float>(R.r17)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) / static_cast<float>(R.r40)));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r38 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r38)));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r38) * static_cast<float>(R.r17)));
        R.r44 = static_cast<float>((-0x1.0000000000000p+0f));
        R.r45 = static_cast<float>((0x0.0p+0f));
        R.r45 = static_cast<float>(op_fma(R.r42, R.r42, R.r45));
        R.r45 = static_cast<float>(op_fma(R.r43, R.r43, R.r45));
        R.r45 = static_cast<float>(op_fma(R.r44, R.r44, R.r45));
        R.r45 = static_cast<float>(op_rsqrt(static_cast<float>(R.r45)));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) * static_cast<float>(R.r45)));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r43) * static_cast<float>(R.r45)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r44) * static_cast<float>(R.r45)));
        R.r46 = static_cast<float>(R.r14);
        R.r47 = static_cast<float>(R.r15);
        R.r48 = static_cast<float>(R.r16);
        R.r49 = static_cast<float>((0x1.0000000000000p+0f));
        R.r50 = static_cast<float>((0x1.0000000000000p+0f));
        R.r51 = static_cast<float>((0x1.0000000000000p+0f));
        R.r3 = static_cast<float>((0x0.0p+0f));
        R.r4 = static_cast<float>((0x0.0p+0f));
        R.r5 = static_cast<float>((0x0.0p+0f));
        R.r52 = static_cast<unsigned int>(((unsigned int)0x0ull));
        goto L_B2;
    L_B2: // bounce
        if(budget == 0u) return 2;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 2, 5u);
        R.r53 = static_cast<float>((0x1.93e5960000000p+99f));
        R.r54 = static_cast<unsigned int>(R.r13);
        R.r55 = static_cast<unsigned int>(((unsigned int)0x0ull));
        R.r56 = static_cast<unsigned int>(R.r12);
        goto L_B3;
    L_B3: // isect
        if(stop_heavy && !fresh) return 3;
    L_B3_again:
        if(budget == 0u) return 3;
        --budget;
    L_B3_spin:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 3, 38u);
        R.r57 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r56)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r58 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r59 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x3ull))));
        R.r60 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r61 = static_cast<float>(static_cast<float>(static_cast<float>(R.r57) - static_cast<float>(R.r46)));
        R.r62 = static_cast<float>(static_cast<float>(static_cast<float>(R.r58) - static_cast<float>(R.r47)));
        R.r63 = static_cast<float>(static_cast<float>(static_cast<float>(R.r59) - static_cast<float>(R.r48)));
        R.r64 = static_cast<float>((0x0.0p+0f));
        R.r64 = static_cast<float>(op_fma(R.r61, R.r42, R.r64));
        R.r64 = static_cast<float>(op_fma(R.r62, R.r43, R.r64));
        R.r64 = static_cast<float>(op_fma(R.r63, R.r44, R.r64));
        R.r65 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r64)));
        R.r66 = static_cast<float>(op_fma(R.r65, R.r42, R.r61));
        R.r67 = static_cast<float>(op_fma(R.r65, R.r43, R.r62));
        R.r68 = static_cast<float>(op_fma(R.r65, R.r44, R.r63));
        R.r69 = static_cast<float>((0x0.0p+0f));
        R.r69 = static_cast<float>(op_fma(R.r66, R.r66, R.r69));
        R.r69 = static_cast<float>(op_fma(R.r67, R.r67, R.r69));
        R.r69 = static_cast<float>(op_fma(R.r68, R.r68, R.r69));
        R.r70 = static_cast<float>(op_fma(R.r60, R.r60, (-(R.r69))));
        R.r71 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r70) >= static_cast<float>((0x0.0p+0f))));
        R.r70 = static_cast<float>(op_max<float>(static_cast<float>(R.r70), static_cast<float>((0x0.0p+0f))));
        R.r72 = static_cast<float>(op_sqrt(static_cast<float>(R.r70)));
        R.r73 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) - static_cast<float>(R.r72)));
        R.r74 = static_cast<float>(static_cast<float>(static_cast<float>(R.r64) + static_cast<float>(R.r72)));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r73) > static_cast<float>((0x1.9999980000000p-5f))));
        R.r75 = static_cast<float>(((R.r33) ? (R.r73) : (R.r74)));
        R.r71 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r71) && static_cast<unsigned int>(static_cast<float>(R.r75) > static_cast<float>((0x1.9999980000000p-5f)))));
        R.r71 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r71) && static_cast<unsigned int>(static_cast<float>(R.r75) < static_cast<float>(R.r53))));
        R.r53 = static_cast<float>(((R.r71) ? (R.r75) : (R.r53)));
        R.r54 = static_cast<unsigned int>(((R.r71) ? (R.r55) : (R.r54)));
        R.r55 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r55) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r56 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r55) < static_cast<unsigned int>(R.r13)));
        if(R.r33) { if(spin != 0u) { --spin; goto L_B3_spin; } goto L_B3_again; } else goto L_B4;
    L_B4: // shade
        fresh = false;
        if constexpr(kProf) count_block(ctx, 4, 2u);
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r54) >= static_cast<unsigned int>(R.r13)));
        if(R.r33) goto L_HALT; else goto L_B5;
    L_B5: // hitp
        if(stop_heavy && !fresh) return 5;
    L_B5_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 5, 28u);
        R.r56 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r54) * static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r56 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(R.r12)));
        R.r57 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r56)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r58 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r59 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x3ull))));
        R.r60 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r76 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r77 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r78 = static_cast<float>(table_load<float>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r8 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r56) + static_cast<unsigned int>(((unsigned int)0x7ull))));
        R.r79 = static_cast<unsigned int>(table_load<unsigned int>(*ctx.cols, static_cast<unsigned>(R.r8)));
        R.r80 = static_cast<float>(op_fma(R.r42, R.r53, R.r46));
        R.r81 = static_cast<float>(op_fma(R.r43, R.r53, R.r47));
        R.r82 = static_cast<float>(op_fma(R.r44, R.r53, R.r48));
        R.r83 = static_cast<float>(static_cast<float>(static_cast<float>(R.r80) - static_cast<float>(R.r57)));
        R.r84 = static_cast<float>(static_cast<float>(static_cast<float>(R.r81) - static_cast<float>(R.r58)));
        R.r85 = static_cast<float>(static_cast<float>(static_cast<float>(R.r82) - static_cast<float>(R.r59)));
        R.r83 = static_cast<float>(static_cast<float>(static_cast<float>(R.r83) / static_cast<float>(R.r60)));
        R.r84 = static_cast<float>(static_cast<float>(static_cast<float>(R.r84) / static_cast<float>(R.r60)));
        R.r85 = static_cast<float>(static_cast<float>(static_cast<float>(R.r85) / static_cast<float>(R.r60)));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r79) == static_cast<unsigned int>(((unsigned int)0x3ull))));
        if(R.r33) goto L_B6; else goto L_B7;
    L_B6: // emit
        fresh = false;
        if constexpr(kProf) count_block(ctx, 6, 4u);
        R.r3 = static_cast<float>(op_fma(R.r49, R.r76, R.r3));
        R.r4 = static_cast<float>(op_fma(R.r50, R.r77, R.r4));
        R.r5 = static_cast<float>(op_fma(R.r51, R.r78, R.r5));
        goto L_HALT;
    L_B7: // surf
        fresh = false;
        if constexpr(kProf) count_block(ctx, 7, 3u);
        R.r52 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r52) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r52) >= static_cast<unsigned int>(((unsigned int)0x10ull))));
        if(R.r33) goto L_HALT; else goto L_B8;
    L_B8: // rrchk
        fresh = false;
        if constexpr(kProf) count_block(ctx, 8, 2u);
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<unsigned int>(R.r52) >= static_cast<unsigned int>(((unsigned int)0x5ull))));
        if(R.r33) goto L_B9; else goto L_B12;
    L_B9: // rr_roll
        fresh = false;
        if constexpr(kProf) count_block(ctx, 9, 2u);
        R.r26 = static_cast<unsigned int>(((unsigned int)0x1ull));
        goto L_B23;
    L_B10: // rr
        fresh = false;
        if constexpr(kProf) count_block(ctx, 10, 4u);
        R.r86 = static_cast<float>(op_max<float>(static_cast<float>(R.r76), static_cast<float>(R.r77)));
        R.r86 = static_cast<float>(op_max<float>(static_cast<float>(R.r86), static_cast<float>(R.r78)));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r130)) < static_cast<float>(R.r86)));
        if(R.r33) goto L_B11; else goto L_HALT;
    L_B11: // rr_keep
        fresh = false;
        if constexpr(kProf) count_block(ctx, 11, 4u);
        R.r76 = static_cast<float>(static_cast<float>(static_cast<float>(R.r76) / static_cast<float>(R.r86)));
        R.r77 = static_cast<float>(static_cast<float>(static_cast<float>(R.r77) / static_cast<float>(R.r86)));
        R.r78 = static_cast<float>(static_cast<float>(static_cast<float>(R.r78) / static_cast<float>(R.r86)));
        goto L_B12;
    L_B12: // scatter
        fresh = false;
        if constexpr(kProf) count_block(ctx, 12, 18u);
        R.r49 = static_cast<float>(static_cast<float>(static_cast<float>(R.r49) * static_cast<float>(R.r76)));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) * static_cast<float>(R.r77)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r78)));
        R.r46 = static_cast<float>(R.r80);
        R.r47 = static_cast<float>(R.r81);
        R.r48 = static_cast<float>(R.r82);
        R.r87 = static_cast<float>((0x0.0p+0f));
        R.r87 = static_cast<float>(op_fma(R.r83, R.r42, R.r87));
        R.r87 = static_cast<float>(op_fma(R.r84, R.r43, R.r87));
        R.r87 = static_cast<float>(op_fma(R.r85, R.r44, R.r87));
        R.r88 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r87) < static_cast<float>((0x0.0p+0f))));
        R.r89 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r83)));
        R.r90 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r84)));
        R.r91 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r85)));
        R.r92 = static_cast<float>(((R.r88) ? (R.r83) : (R.r89)));
        R.r93 = static_cast<float>(((R.r88) ? (R.r84) : (R.r90)));
        R.r94 = static_cast<float>(((R.r88) ? (R.r85) : (R.r91)));
        switch(R.r79) {
        case 0: goto L_B14;
        case 1: goto L_B13;
        case 2: goto L_B18;
        default: goto L_HALT;
        }
    L_B13: // mirror
        fresh = false;
        if constexpr(kProf) count_block(ctx, 13, 5u);
        R.r95 = static_cast<float>(static_cast<float>(static_cast<float>(R.r87) * static_cast<float>((-0x1.0000000000000p+1f))));
        R.r42 = static_cast<float>(op_fma(R.r95, R.r83, R.r42));
        R.r43 = static_cast<float>(op_fma(R.r95, R.r84, R.r43));
        R.r44 = static_cast<float>(op_fma(R.r95, R.r85, R.r44));
        goto L_B2;
    L_B14: // diffuse
        if(stop_heavy && !fresh) return 14;
    L_B14_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 14, 26u);
        R.r96 = static_cast<float>(op_abs(static_cast<float>(R.r92)));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r96) > static_cast<float>((0x1.99999a0000000p-4f))));
        R.r97 = static_cast<float>(((R.r33) ? ((0x0.0p+0f)) : ((0x1.0000000000000p+0f))));
        R.r98 = static_cast<float>(((R.r33) ? ((0x1.0000000000000p+0f)) : ((0x0.0p+0f))));
        R.r99 = static_cast<float>((0x0.0p+0f));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r99) * static_cast<float>(R.r93)));
        R.r100 = static_cast<float>(op_fma(R.r98, R.r94, (-(R.r45))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r97) * static_cast<float>(R.r94)));
        R.r101 = static_cast<float>(op_fma(R.r99, R.r92, (-(R.r45))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r98) * static_cast<float>(R.r92)));
        R.r102 = static_cast<float>(op_fma(R.r97, R.r93, (-(R.r45))));
        R.r45 = static_cast<float>((0x0.0p+0f));
        R.r45 = static_cast<float>(op_fma(R.r100, R.r100, R.r45));
        R.r45 = static_cast<float>(op_fma(R.r101, R.r101, R.r45));
        R.r45 = static_cast<float>(op_fma(R.r102, R.r102, R.r45));
        R.r45 = static_cast<float>(op_rsqrt(static_cast<float>(R.r45)));
        R.r100 = static_cast<float>(static_cast<float>(static_cast<float>(R.r100) * static_cast<float>(R.r45)));
        R.r101 = static_cast<float>(static_cast<float>(static_cast<float>(R.r101) * static_cast<float>(R.r45)));
        R.r102 = static_cast<float>(static_cast<float>(static_cast<float>(R.r102) * static_cast<float>(R.r45)));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r94) * static_cast<float>(R.r101)));
        R.r103 = static_cast<float>(op_fma(R.r93, R.r102, (-(R.r45))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r92) * static_cast<float>(R.r102)));
        R.r104 = static_cast<float>(op_fma(R.r94, R.r100, (-(R.r45))));
        R.r45 = static_cast<float>(static_cast<float>(static_cast<float>(R.r93) * static_cast<float>(R.r100)));
        R.r105 = static_cast<float>(op_fma(R.r92, R.r101, (-(R.r45))));
        goto L_B15;
    L_B15: // disk_roll
        fresh = false;
        if constexpr(kProf) count_block(ctx, 15, 2u);
        R.r26 = static_cast<unsigned int>(((unsigned int)0x2ull));
        goto L_B23;
    L_B16: // disk
        fresh = false;
        if constexpr(kProf) count_block(ctx, 16, 8u);
        R.r106 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r130)) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r106 = static_cast<float>(static_cast<float>(static_cast<float>(R.r106) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r107 = static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r131)) * static_cast<float>((0x1.0000000000000p+1f))));
        R.r107 = static_cast<float>(static_cast<float>(static_cast<float>(R.r107) - static_cast<float>((0x1.0000000000000p+0f))));
        R.r108 = static_cast<float>(static_cast<float>(static_cast<float>(R.r106) * static_cast<float>(R.r106)));
        R.r108 = static_cast<float>(op_fma(R.r107, R.r107, R.r108));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r108) < static_cast<float>((0x1.0000000000000p+0f))));
        if(R.r33) goto L_B17; else goto L_B15;
    L_B17: // disk_ok
        fresh = false;
        if constexpr(kProf) count_block(ctx, 17, 20u);
        R.r109 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r108)));
        R.r109 = static_cast<float>(op_sqrt(static_cast<float>(R.r109)));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r100) * static_cast<float>(R.r106)));
        R.r42 = static_cast<float>(op_fma(R.r103, R.r107, R.r42));
        R.r42 = static_cast<float>(op_fma(R.r92, R.r109, R.r42));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r101) * static_cast<float>(R.r106)));
        R.r43 = static_cast<float>(op_fma(R.r104, R.r107, R.r43));
        R.r43 = static_cast<float>(op_fma(R.r93, R.r109, R.r43));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r102) * static_cast<float>(R.r106)));
        R.r44 = static_cast<float>(op_fma(R.r105, R.r107, R.r44));
        R.r44 = static_cast<float>(op_fma(R.r94, R.r109, R.r44));
        R.r45 = static_cast<float>((0x0.0p+0f));
        R.r45 = static_cast<float>(op_fma(R.r42, R.r42, R.r45));
        R.r45 = static_cast<float>(op_fma(R.r43, R.r43, R.r45));
        R.r45 = static_cast<float>(op_fma(R.r44, R.r44, R.r45));
        R.r45 = static_cast<float>(op_rsqrt(static_cast<float>(R.r45)));
        R.r42 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) * static_cast<float>(R.r45)));
        R.r43 = static_cast<float>(static_cast<float>(static_cast<float>(R.r43) * static_cast<float>(R.r45)));
        R.r44 = static_cast<float>(static_cast<float>(static_cast<float>(R.r44) * static_cast<float>(R.r45)));
        goto L_B2;
    L_B18: // glass
        fresh = false;
        if constexpr(kProf) count_block(ctx, 18, 13u);
        R.r110 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) / static_cast<float>((0x1.8000000000000p+0f))));
        R.r111 = static_cast<float>(((R.r88) ? (R.r110) : ((0x1.8000000000000p+0f))));
        R.r112 = static_cast<float>((0x0.0p+0f));
        R.r112 = static_cast<float>(op_fma(R.r42, R.r92, R.r112));
        R.r112 = static_cast<float>(op_fma(R.r43, R.r93, R.r112));
        R.r112 = static_cast<float>(op_fma(R.r44, R.r94, R.r112));
        R.r113 = static_cast<float>(static_cast<float>(static_cast<float>(R.r112) * static_cast<float>(R.r112)));
        R.r113 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r113)));
        R.r114 = static_cast<float>(static_cast<float>(static_cast<float>(R.r111) * static_cast<float>(R.r111)));
        R.r113 = static_cast<float>(static_cast<float>(static_cast<float>(R.r113) * static_cast<float>(R.r114)));
        R.r113 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r113)));
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(R.r113) < static_cast<float>((0x0.0p+0f))));
        if(R.r33) goto L_B13; else goto L_B19;
    L_B19: // refr
        if(stop_heavy && !fresh) return 19;
    L_B19_again:
        fresh = false;
        if constexpr(kProf) count_block(ctx, 19, 40u);
        R.r115 = static_cast<float>(op_sqrt(static_cast<float>(R.r113)));
        R.r115 = static_cast<float>(op_fma(R.r112, R.r111, R.r115));
        R.r116 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r115)));
        R.r115 = static_cast<float>(((R.r88) ? (R.r115) : (R.r116)));
        R.r116 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r115)));
        R.r117 = static_cast<float>(static_cast<float>(static_cast<float>(R.r42) * static_cast<float>(R.r111)));
        R.r117 = static_cast<float>(op_fma(R.r116, R.r83, R.r117));
        R.r118 = static_cast<float>(static_cast<float>(static_cast<float>(R.r43) * static_cast<float>(R.r111)));
        R.r118 = static_cast<float>(op_fma(R.r116, R.r84, R.r118));
        R.r119 = static_cast<float>(static_cast<float>(static_cast<float>(R.r44) * static_cast<float>(R.r111)));
        R.r119 = static_cast<float>(op_fma(R.r116, R.r85, R.r119));
        R.r45 = static_cast<float>((0x0.0p+0f));
        R.r45 = static_cast<float>(op_fma(R.r117, R.r117, R.r45));
        R.r45 = static_cast<float>(op_fma(R.r118, R.r118, R.r45));
        R.r45 = static_cast<float>(op_fma(R.r119, R.r119, R.r45));
        R.r45 = static_cast<float>(op_rsqrt(static_cast<float>(R.r45)));
        R.r117 = static_cast<float>(static_cast<float>(static_cast<float>(R.r117) * static_cast<float>(R.r45)));
        R.r118 = static_cast<float>(static_cast<float>(static_cast<float>(R.r118) * static_cast<float>(R.r45)));
        R.r119 = static_cast<float>(static_cast<float>(static_cast<float>(R.r119) * static_cast<float>(R.r45)));
        R.r120 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p-1f)) / static_cast<float>((0x1.4000000000000p+1f))));
        R.r120 = static_cast<float>(static_cast<float>(static_cast<float>(R.r120) * static_cast<float>(R.r120)));
        R.r121 = static_cast<float>((0x0.0p+0f));
        R.r121 = static_cast<float>(op_fma(R.r117, R.r83, R.r121));
        R.r121 = static_cast<float>(op_fma(R.r118, R.r84, R.r121));
        R.r121 = static_cast<float>(op_fma(R.r119, R.r85, R.r121));
        R.r122 = static_cast<float>(static_cast<float>(-static_cast<float>(R.r112)));
        R.r123 = static_cast<float>(((R.r88) ? (R.r122) : (R.r121)));
        R.r123 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r123)));
        R.r124 = static_cast<float>(static_cast<float>(static_cast<float>(R.r123) * static_cast<float>(R.r123)));
        R.r124 = static_cast<float>(static_cast<float>(static_cast<float>(R.r124) * static_cast<float>(R.r124)));
        R.r124 = static_cast<float>(static_cast<float>(static_cast<float>(R.r124) * static_cast<float>(R.r123)));
        R.r125 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r120)));
        R.r125 = static_cast<float>(op_fma(R.r125, R.r124, R.r120));
        R.r126 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r125)));
        R.r127 = static_cast<float>(op_fma(R.r125, (0x1.0000000000000p-1f), (0x1.0000000000000p-2f)));
        R.r128 = static_cast<float>(static_cast<float>(static_cast<float>(R.r125) / static_cast<float>(R.r127)));
        R.r129 = static_cast<float>(static_cast<float>(static_cast<float>((0x1.0000000000000p+0f)) - static_cast<float>(R.r127)));
        R.r129 = static_cast<float>(static_cast<float>(static_cast<float>(R.r126) / static_cast<float>(R.r129)));
        R.r26 = static_cast<unsigned int>(((unsigned int)0x3ull));
        goto L_B23;
    L_B20: // fres
        fresh = false;
        if constexpr(kProf) count_block(ctx, 20, 2u);
        R.r33 = static_cast<unsigned int>(static_cast<bool>(static_cast<float>(bitcast<float>(R.r130)) < static_cast<float>(R.r127)));
        if(R.r33) goto L_B21; else goto L_B22;
    L_B21: // take_refl
        fresh = false;
        if constexpr(kProf) count_block(ctx, 21, 4u);
        R.r49 = static_cast<float>(static_cast<float>(static_cast<float>(R.r49) * static_cast<float>(R.r128)));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) * static_cast<float>(R.r128)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r128)));
        goto L_B13;
    L_B22: // take_refr
        fresh = false;
        if constexpr(kProf) count_block(ctx, 22, 7u);
        R.r49 = static_cast<float>(static_cast<float>(static_cast<float>(R.r49) * static_cast<float>(R.r129)));
        R.r50 = static_cast<float>(static_cast<float>(static_cast<float>(R.r50) * static_cast<float>(R.r129)));
        R.r51 = static_cast<float>(static_cast<float>(static_cast<float>(R.r51) * static_cast<float>(R.r129)));
        R.r42 = static_cast<float>(R.r117);
        R.r43 = static_cast<float>(R.r118);
        R.r44 = static_cast<float>(R.r119);
        goto L_B2;
    L_B23: // roll
        if(stop_heavy && !fresh) return 23;
    L_B23_again:
        if(budget == 0u) return 23;
        --budget;
        fresh = false;
        if constexpr(kProf) count_block(ctx, 23, 292u);
        R.r130 = static_cast<unsigned int>(R.r24);
        R.r131 = static_cast<unsigned int>(R.r25);
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r11)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x9e3779b9ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(((unsigned int)0x9e3779b9ull))));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(R.r23)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r23)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(R.r11)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x2ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r11)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x9e3779b9ull))));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x3ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(((unsigned int)0x9e3779b9ull))));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(R.r23)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x4ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r23)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(R.r11)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x5ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r11)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x9e3779b9ull))));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xdull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xdull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0xfull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0xfull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1aull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1aull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x6ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x6ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(((unsigned int)0x9e3779b9ull))));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(R.r23)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x7ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x11ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x11ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x1dull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x1dull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x10ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x10ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r131)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x18ull)) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) << static_cast<unsigned int>(R.r132)));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(((unsigned int)0x20ull)) - static_cast<unsigned int>(((unsigned int)0x18ull))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r133) & static_cast<unsigned int>(((unsigned int)0x1full))));
        R.r133 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(R.r133)));
        R.r132 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) | static_cast<unsigned int>(R.r133)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r132) ^ static_cast<unsigned int>(R.r130)));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) + static_cast<unsigned int>(R.r23)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(R.r11)));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) + static_cast<unsigned int>(((unsigned int)0x8ull))));
        R.r25 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r25) + static_cast<unsigned int>(((unsigned int)0x1ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) >> static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r130 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r130) | static_cast<unsigned int>(((unsigned int)0x3f800000ull))));
        R.r130 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r130)) - static_cast<float>((0x1.0000000000000p+0f)))));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) >> static_cast<unsigned int>(((unsigned int)0x9ull))));
        R.r131 = static_cast<unsigned int>(static_cast<unsigned int>(static_cast<unsigned int>(R.r131) | static_cast<unsigned int>(((unsigned int)0x3f800000ull))));
        R.r131 = bitcast<unsigned int>(static_cast<float>(static_cast<float>(static_cast<float>(bitcast<float>(R.r131)) - static_cast<float>((0x1.0000000000000p+0f)))));
        switch(R.r26) {
        case 0: goto L_B1;
        case 1: goto L_B10;
        case 2: goto L_B16;
        case 3: goto L_B20;
        default: goto L_HALT;
        }
    L_HALT:
        return kHalt;
    }

    static constexpr unsigned long long kRowBytes = 2832ull;
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
                v0.y = bitcast<unsigned>(R.r2);
                v0.z = tid;
                reinterpret_cast<uint4*>(base + 0ull * cap)[idx] = v0;
            }
            return;
        }
        case 1: // prim
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r7);
                v0.y = bitcast<unsigned>(R.r9);
                v0.z = bitcast<unsigned>(R.r11);
                v0.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 16ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r13);
                v1.y = bitcast<unsigned>(R.r14);
                v1.z = bitcast<unsigned>(R.r15);
                v1.w = bitcast<unsigned>(R.r16);
                reinterpret_cast<uint4*>(base + 32ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r17);
                v2.y = bitcast<unsigned>(R.r20);
                v2.z = bitcast<unsigned>(R.r21);
                v2.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 48ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r23);
                v3.y = bitcast<unsigned>(R.r24);
                v3.z = bitcast<unsigned>(R.r25);
                v3.w = bitcast<unsigned>(R.r130);
                reinterpret_cast<uint4*>(base + 64ull * cap)[idx] = v3;
            }
            {
                uint2 v4;
                v4.x = bitcast<unsigned>(R.r131);
                v4.y = tid;
                reinterpret_cast<uint2*>(base + 80ull * cap)[idx] = v4;
            }
            return;
        }
        case 2: // bounce
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 88ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 104ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 120ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 136ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = tid;
                reinterpret_cast<uint4*>(base + 152ull * cap)[idx] = v4;
            }
            return;
        }
        case 3: // isect
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 168ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 184ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 200ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 216ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = bitcast<unsigned>(R.r53);
                reinterpret_cast<uint4*>(base + 232ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r54);
                v5.y = bitcast<unsigned>(R.r55);
                v5.z = bitcast<unsigned>(R.r56);
                v5.w = tid;
                reinterpret_cast<uint4*>(base + 248ull * cap)[idx] = v5;
            }
            return;
        }
        case 4: // shade
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 264ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 280ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 296ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 312ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = bitcast<unsigned>(R.r53);
                reinterpret_cast<uint4*>(base + 328ull * cap)[idx] = v4;
            }
            {
                uint2 v5;
                v5.x = bitcast<unsigned>(R.r54);
                v5.y = tid;
                reinterpret_cast<uint2*>(base + 344ull * cap)[idx] = v5;
            }
            return;
        }
        case 5: // hitp
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 352ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 368ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 384ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 400ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = bitcast<unsigned>(R.r53);
                reinterpret_cast<uint4*>(base + 416ull * cap)[idx] = v4;
            }
            {
                uint2 v5;
                v5.x = bitcast<unsigned>(R.r54);
                v5.y = tid;
                reinterpret_cast<uint2*>(base + 432ull * cap)[idx] = v5;
            }
            return;
        }
        case 6: // emit
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 440ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r50);
                v1.y = bitcast<unsigned>(R.r51);
                v1.z = bitcast<unsigned>(R.r76);
                v1.w = bitcast<unsigned>(R.r77);
                reinterpret_cast<uint4*>(base + 456ull * cap)[idx] = v1;
            }
            {
                uint2 v2;
                v2.x = bitcast<unsigned>(R.r78);
                v2.y = tid;
                reinterpret_cast<uint2*>(base + 472ull * cap)[idx] = v2;
            }
            return;
        }
        case 7: // surf
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 480ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 496ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 512ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 528ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r76);
                v4.y = bitcast<unsigned>(R.r77);
                v4.z = bitcast<unsigned>(R.r78);
                v4.w = bitcast<unsigned>(R.r79);
                reinterpret_cast<uint4*>(base + 544ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r80);
                v5.y = bitcast<unsigned>(R.r81);
                v5.z = bitcast<unsigned>(R.r82);
                v5.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 560ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r84);
                v6.y = bitcast<unsigned>(R.r85);
                v6.z = tid;
                reinterpret_cast<uint4*>(base + 576ull * cap)[idx] = v6;
            }
            return;
        }
        case 8: // rrchk
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 592ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 608ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 624ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 640ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r76);
                v4.y = bitcast<unsigned>(R.r77);
                v4.z = bitcast<unsigned>(R.r78);
                v4.w = bitcast<unsigned>(R.r79);
                reinterpret_cast<uint4*>(base + 656ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r80);
                v5.y = bitcast<unsigned>(R.r81);
                v5.z = bitcast<unsigned>(R.r82);
                v5.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 672ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r84);
                v6.y = bitcast<unsigned>(R.r85);
                v6.z = tid;
                reinterpret_cast<uint4*>(base + 688ull * cap)[idx] = v6;
            }
            return;
        }
        case 9: // rr_roll
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 704ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 720ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 736ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 752ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r76);
                v4.y = bitcast<unsigned>(R.r77);
                v4.z = bitcast<unsigned>(R.r78);
                v4.w = bitcast<unsigned>(R.r79);
                reinterpret_cast<uint4*>(base + 768ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r80);
                v5.y = bitcast<unsigned>(R.r81);
                v5.z = bitcast<unsigned>(R.r82);
                v5.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 784ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r84);
                v6.y = bitcast<unsigned>(R.r85);
                v6.z = tid;
                reinterpret_cast<uint4*>(base + 800ull * cap)[idx] = v6;
            }
            return;
        }
        case 10: // rr
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 816ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 832ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 848ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 864ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r76);
                v4.y = bitcast<unsigned>(R.r77);
                v4.z = bitcast<unsigned>(R.r78);
                v4.w = bitcast<unsigned>(R.r79);
                reinterpret_cast<uint4*>(base + 880ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r80);
                v5.y = bitcast<unsigned>(R.r81);
                v5.z = bitcast<unsigned>(R.r82);
                v5.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 896ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r84);
                v6.y = bitcast<unsigned>(R.r85);
                v6.z = bitcast<unsigned>(R.r130);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 912ull * cap)[idx] = v6;
            }
            return;
        }
        case 11: // rr_keep
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 928ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 944ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 960ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 976ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r76);
                v4.y = bitcast<unsigned>(R.r77);
                v4.z = bitcast<unsigned>(R.r78);
                v4.w = bitcast<unsigned>(R.r79);
                reinterpret_cast<uint4*>(base + 992ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r80);
                v5.y = bitcast<unsigned>(R.r81);
                v5.z = bitcast<unsigned>(R.r82);
                v5.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 1008ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r84);
                v6.y = bitcast<unsigned>(R.r85);
                v6.z = bitcast<unsigned>(R.r86);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 1024ull * cap)[idx] = v6;
            }
            return;
        }
        case 12: // scatter
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 1040ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1056ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 1072ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 1088ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r76);
                v4.y = bitcast<unsigned>(R.r77);
                v4.z = bitcast<unsigned>(R.r78);
                v4.w = bitcast<unsigned>(R.r79);
                reinterpret_cast<uint4*>(base + 1104ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r80);
                v5.y = bitcast<unsigned>(R.r81);
                v5.z = bitcast<unsigned>(R.r82);
                v5.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 1120ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r84);
                v6.y = bitcast<unsigned>(R.r85);
                v6.z = tid;
                reinterpret_cast<uint4*>(base + 1136ull * cap)[idx] = v6;
            }
            return;
        }
        case 13: // mirror
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 1152ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1168ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 1184ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 1200ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 1216ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r84);
                v5.y = bitcast<unsigned>(R.r85);
                v5.z = bitcast<unsigned>(R.r87);
                v5.w = tid;
                reinterpret_cast<uint4*>(base + 1232ull * cap)[idx] = v5;
            }
            return;
        }
        case 14: // diffuse
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 1248ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1264ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r46);
                v2.z = bitcast<unsigned>(R.r47);
                v2.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 1280ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 1296ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r92);
                v4.y = bitcast<unsigned>(R.r93);
                v4.z = bitcast<unsigned>(R.r94);
                v4.w = tid;
                reinterpret_cast<uint4*>(base + 1312ull * cap)[idx] = v4;
            }
            return;
        }
        case 15: // disk_roll
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 1328ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1344ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r46);
                v2.z = bitcast<unsigned>(R.r47);
                v2.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 1360ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 1376ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r92);
                v4.y = bitcast<unsigned>(R.r93);
                v4.z = bitcast<unsigned>(R.r94);
                v4.w = bitcast<unsigned>(R.r100);
                reinterpret_cast<uint4*>(base + 1392ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r101);
                v5.y = bitcast<unsigned>(R.r102);
                v5.z = bitcast<unsigned>(R.r103);
                v5.w = bitcast<unsigned>(R.r104);
                reinterpret_cast<uint4*>(base + 1408ull * cap)[idx] = v5;
            }
            {
                uint2 v6;
                v6.x = bitcast<unsigned>(R.r105);
                v6.y = tid;
                reinterpret_cast<uint2*>(base + 1424ull * cap)[idx] = v6;
            }
            return;
        }
        case 16: // disk
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 1432ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1448ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r46);
                v2.z = bitcast<unsigned>(R.r47);
                v2.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 1464ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 1480ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r92);
                v4.y = bitcast<unsigned>(R.r93);
                v4.z = bitcast<unsigned>(R.r94);
                v4.w = bitcast<unsigned>(R.r100);
                reinterpret_cast<uint4*>(base + 1496ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r101);
                v5.y = bitcast<unsigned>(R.r102);
                v5.z = bitcast<unsigned>(R.r103);
                v5.w = bitcast<unsigned>(R.r104);
                reinterpret_cast<uint4*>(base + 1512ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r105);
                v6.y = bitcast<unsigned>(R.r130);
                v6.z = bitcast<unsigned>(R.r131);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 1528ull * cap)[idx] = v6;
            }
            return;
        }
        case 17: // disk_ok
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 1544ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1560ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r46);
                v2.z = bitcast<unsigned>(R.r47);
                v2.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 1576ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 1592ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r92);
                v4.y = bitcast<unsigned>(R.r93);
                v4.z = bitcast<unsigned>(R.r94);
                v4.w = bitcast<unsigned>(R.r100);
                reinterpret_cast<uint4*>(base + 1608ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r101);
                v5.y = bitcast<unsigned>(R.r102);
                v5.z = bitcast<unsigned>(R.r103);
                v5.w = bitcast<unsigned>(R.r104);
                reinterpret_cast<uint4*>(base + 1624ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r105);
                v6.y = bitcast<unsigned>(R.r106);
                v6.z = bitcast<unsigned>(R.r107);
                v6.w = bitcast<unsigned>(R.r108);
                reinterpret_cast<uint4*>(base + 1640ull * cap)[idx] = v6;
            }
            {
                unsigned v7;
                v7 = tid;
                reinterpret_cast<unsigned*>(base + 1656ull * cap)[idx] = v7;
            }
            return;
        }
        case 18: // glass
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 1664ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1680ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 1696ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 1712ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 1728ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r84);
                v5.y = bitcast<unsigned>(R.r85);
                v5.z = bitcast<unsigned>(R.r87);
                v5.w = bitcast<unsigned>(R.r88);
                reinterpret_cast<uint4*>(base + 1744ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r92);
                v6.y = bitcast<unsigned>(R.r93);
                v6.z = bitcast<unsigned>(R.r94);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 1760ull * cap)[idx] = v6;
            }
            return;
        }
        case 19: // refr
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 1776ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1792ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 1808ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 1824ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 1840ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r84);
                v5.y = bitcast<unsigned>(R.r85);
                v5.z = bitcast<unsigned>(R.r87);
                v5.w = bitcast<unsigned>(R.r88);
                reinterpret_cast<uint4*>(base + 1856ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r111);
                v6.y = bitcast<unsigned>(R.r112);
                v6.z = bitcast<unsigned>(R.r113);
                v6.w = tid;
                reinterpret_cast<uint4*>(base + 1872ull * cap)[idx] = v6;
            }
            return;
        }
        case 20: // fres
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 1888ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 1904ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 1920ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 1936ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 1952ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r84);
                v5.y = bitcast<unsigned>(R.r85);
                v5.z = bitcast<unsigned>(R.r87);
                v5.w = bitcast<unsigned>(R.r117);
                reinterpret_cast<uint4*>(base + 1968ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r118);
                v6.y = bitcast<unsigned>(R.r119);
                v6.z = bitcast<unsigned>(R.r127);
                v6.w = bitcast<unsigned>(R.r128);
                reinterpret_cast<uint4*>(base + 1984ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r129);
                v7.y = bitcast<unsigned>(R.r130);
                v7.z = tid;
                reinterpret_cast<uint4*>(base + 2000ull * cap)[idx] = v7;
            }
            return;
        }
        case 21: // take_refl
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 2016ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 2032ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 2048ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 2064ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 2080ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r84);
                v5.y = bitcast<unsigned>(R.r85);
                v5.z = bitcast<unsigned>(R.r87);
                v5.w = bitcast<unsigned>(R.r128);
                reinterpret_cast<uint4*>(base + 2096ull * cap)[idx] = v5;
            }
            {
                unsigned v6;
                v6 = tid;
                reinterpret_cast<unsigned*>(base + 2112ull * cap)[idx] = v6;
            }
            return;
        }
        case 22: // take_refr
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 2120ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 2136ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r46);
                v2.z = bitcast<unsigned>(R.r47);
                v2.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 2152ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 2168ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r117);
                v4.y = bitcast<unsigned>(R.r118);
                v4.z = bitcast<unsigned>(R.r119);
                v4.w = bitcast<unsigned>(R.r129);
                reinterpret_cast<uint4*>(base + 2184ull * cap)[idx] = v4;
            }
            {
                unsigned v5;
                v5 = tid;
                reinterpret_cast<unsigned*>(base + 2200ull * cap)[idx] = v5;
            }
            return;
        }
        case 23: // roll
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r7);
                reinterpret_cast<uint4*>(base + 2208ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r9);
                v1.y = bitcast<unsigned>(R.r11);
                v1.z = bitcast<unsigned>(R.r12);
                v1.w = bitcast<unsigned>(R.r13);
                reinterpret_cast<uint4*>(base + 2224ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r14);
                v2.y = bitcast<unsigned>(R.r15);
                v2.z = bitcast<unsigned>(R.r16);
                v2.w = bitcast<unsigned>(R.r17);
                reinterpret_cast<uint4*>(base + 2240ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r20);
                v3.y = bitcast<unsigned>(R.r21);
                v3.z = bitcast<unsigned>(R.r22);
                v3.w = bitcast<unsigned>(R.r23);
                reinterpret_cast<uint4*>(base + 2256ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r24);
                v4.y = bitcast<unsigned>(R.r25);
                v4.z = bitcast<unsigned>(R.r26);
                v4.w = bitcast<unsigned>(R.r42);
                reinterpret_cast<uint4*>(base + 2272ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r43);
                v5.y = bitcast<unsigned>(R.r44);
                v5.z = bitcast<unsigned>(R.r46);
                v5.w = bitcast<unsigned>(R.r47);
                reinterpret_cast<uint4*>(base + 2288ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r48);
                v6.y = bitcast<unsigned>(R.r49);
                v6.z = bitcast<unsigned>(R.r50);
                v6.w = bitcast<unsigned>(R.r51);
                reinterpret_cast<uint4*>(base + 2304ull * cap)[idx] = v6;
            }
            {
                uint4 v7;
                v7.x = bitcast<unsigned>(R.r52);
                v7.y = bitcast<unsigned>(R.r76);
                v7.z = bitcast<unsigned>(R.r77);
                v7.w = bitcast<unsigned>(R.r78);
                reinterpret_cast<uint4*>(base + 2320ull * cap)[idx] = v7;
            }
            {
                uint4 v8;
                v8.x = bitcast<unsigned>(R.r79);
                v8.y = bitcast<unsigned>(R.r80);
                v8.z = bitcast<unsigned>(R.r81);
                v8.w = bitcast<unsigned>(R.r82);
                reinterpret_cast<uint4*>(base + 2336ull * cap)[idx] = v8;
            }
            {
                uint4 v9;
                v9.x = bitcast<unsigned>(R.r83);
                v9.y = bitcast<unsigned>(R.r84);
                v9.z = bitcast<unsigned>(R.r85);
                v9.w = bitcast<unsigned>(R.r87);
                reinterpret_cast<uint4*>(base + 2352ull * cap)[idx] = v9;
            }
            {
                uint4 v10;
                v10.x = bitcast<unsigned>(R.r92);
                v10.y = bitcast<unsigned>(R.r93);
                v10.z = bitcast<unsigned>(R.r94);
                v10.w = bitcast<unsigned>(R.r100);
                reinterpret_cast<uint4*>(base + 2368ull * cap)[idx] = v10;
            }
            {
                uint4 v11;
                v11.x = bitcast<unsigned>(R.r101);
                v11.y = bitcast<unsigned>(R.r102);
                v11.z = bitcast<unsigned>(R.r103);
                v11.w = bitcast<unsigned>(R.r104);
                reinterpret_cast<uint4*>(base + 2384ull * cap)[idx] = v11;
            }
            {
                uint4 v12;
                v12.x = bitcast<unsigned>(R.r105);
                v12.y = bitcast<unsigned>(R.r117);
                v12.z = bitcast<unsigned>(R.r118);
                v12.w = bitcast<unsigned>(R.r119);
                reinterpret_cast<uint4*>(base + 2400ull * cap)[idx] = v12;
            }
            {
                uint4 v13;
                v13.x = bitcast<unsigned>(R.r127);
                v13.y = bitcast<unsigned>(R.r128);
                v13.z = bitcast<unsigned>(R.r129);
                v13.w = tid;
                reinterpret_cast<uint4*>(base + 2416ull * cap)[idx] = v13;
            }
            return;
        }
        case 24: // roll, context 0
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r7);
                v0.y = bitcast<unsigned>(R.r9);
                v0.z = bitcast<unsigned>(R.r11);
                v0.w = bitcast<unsigned>(R.r12);
                reinterpret_cast<uint4*>(base + 2432ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r13);
                v1.y = bitcast<unsigned>(R.r14);
                v1.z = bitcast<unsigned>(R.r15);
                v1.w = bitcast<unsigned>(R.r16);
                reinterpret_cast<uint4*>(base + 2448ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r17);
                v2.y = bitcast<unsigned>(R.r20);
                v2.z = bitcast<unsigned>(R.r21);
                v2.w = bitcast<unsigned>(R.r22);
                reinterpret_cast<uint4*>(base + 2464ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r23);
                v3.y = bitcast<unsigned>(R.r24);
                v3.z = bitcast<unsigned>(R.r25);
                v3.w = tid;
                reinterpret_cast<uint4*>(base + 2480ull * cap)[idx] = v3;
            }
            return;
        }
        case 25: // roll, context 1
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 2496ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 2512ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 2528ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 2544ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r76);
                v4.y = bitcast<unsigned>(R.r77);
                v4.z = bitcast<unsigned>(R.r78);
                v4.w = bitcast<unsigned>(R.r79);
                reinterpret_cast<uint4*>(base + 2560ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r80);
                v5.y = bitcast<unsigned>(R.r81);
                v5.z = bitcast<unsigned>(R.r82);
                v5.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 2576ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r84);
                v6.y = bitcast<unsigned>(R.r85);
                v6.z = tid;
                reinterpret_cast<uint4*>(base + 2592ull * cap)[idx] = v6;
            }
            return;
        }
        case 26: // roll, context 2
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 2608ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 2624ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r46);
                v2.z = bitcast<unsigned>(R.r47);
                v2.w = bitcast<unsigned>(R.r48);
                reinterpret_cast<uint4*>(base + 2640ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r49);
                v3.y = bitcast<unsigned>(R.r50);
                v3.z = bitcast<unsigned>(R.r51);
                v3.w = bitcast<unsigned>(R.r52);
                reinterpret_cast<uint4*>(base + 2656ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r92);
                v4.y = bitcast<unsigned>(R.r93);
                v4.z = bitcast<unsigned>(R.r94);
                v4.w = bitcast<unsigned>(R.r100);
                reinterpret_cast<uint4*>(base + 2672ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r101);
                v5.y = bitcast<unsigned>(R.r102);
                v5.z = bitcast<unsigned>(R.r103);
                v5.w = bitcast<unsigned>(R.r104);
                reinterpret_cast<uint4*>(base + 2688ull * cap)[idx] = v5;
            }
            {
                uint2 v6;
                v6.x = bitcast<unsigned>(R.r105);
                v6.y = tid;
                reinterpret_cast<uint2*>(base + 2704ull * cap)[idx] = v6;
            }
            return;
        }
        case 27: // roll, context 3
        {
            {
                uint4 v0;
                v0.x = bitcast<unsigned>(R.r3);
                v0.y = bitcast<unsigned>(R.r4);
                v0.z = bitcast<unsigned>(R.r5);
                v0.w = bitcast<unsigned>(R.r11);
                reinterpret_cast<uint4*>(base + 2712ull * cap)[idx] = v0;
            }
            {
                uint4 v1;
                v1.x = bitcast<unsigned>(R.r12);
                v1.y = bitcast<unsigned>(R.r13);
                v1.z = bitcast<unsigned>(R.r23);
                v1.w = bitcast<unsigned>(R.r24);
                reinterpret_cast<uint4*>(base + 2728ull * cap)[idx] = v1;
            }
            {
                uint4 v2;
                v2.x = bitcast<unsigned>(R.r25);
                v2.y = bitcast<unsigned>(R.r42);
                v2.z = bitcast<unsigned>(R.r43);
                v2.w = bitcast<unsigned>(R.r44);
                reinterpret_cast<uint4*>(base + 2744ull * cap)[idx] = v2;
            }
            {
                uint4 v3;
                v3.x = bitcast<unsigned>(R.r46);
                v3.y = bitcast<unsigned>(R.r47);
                v3.z = bitcast<unsigned>(R.r48);
                v3.w = bitcast<unsigned>(R.r49);
                reinterpret_cast<uint4*>(base + 2760ull * cap)[idx] = v3;
            }
            {
                uint4 v4;
                v4.x = bitcast<unsigned>(R.r50);
                v4.y = bitcast<unsigned>(R.r51);
                v4.z = bitcast<unsigned>(R.r52);
                v4.w = bitcast<unsigned>(R.r83);
                reinterpret_cast<uint4*>(base + 2776ull * cap)[idx] = v4;
            }
            {
                uint4 v5;
                v5.x = bitcast<unsigned>(R.r84);
                v5.y = bitcast<unsigned>(R.r85);
                v5.z = bitcast<unsigned>(R.r87);
                v5.w = bitcast<unsigned>(R.r117);
                reinterpret_cast<uint4*>(base + 2792ull * cap)[idx] = v5;
            }
            {
                uint4 v6;
                v6.x = bitcast<unsigned>(R.r118);
                v6.y = bitcast<unsigned>(R.r119);
                v6.z = bitcast<unsigned>(R.r127);
                v6.w = bitcast<unsigned>(R.r128);
                reinterpret_cast<uint4*>(base + 2808ull * cap)[idx] = v6;
            }
            {
                uint2 v7;
                v7.x = bitcast<unsigned>(R.r129);
                v7.y = tid;
                reinterpret_cast<uint2*>(base + 2824ull * cap)[idx] = v7;
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
            R.r2 = bitcast<unsigned int>(v0.y);
            return v0.z;
        }
        case 1: // prim
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 16ull * cap)[idx];
            R.r7 = bitcast<unsigned int>(v0.x);
            R.r9 = bitcast<unsigned int>(v0.y);
            R.r11 = bitcast<unsigned int>(v0.z);
            R.r12 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 32ull * cap)[idx];
            R.r13 = bitcast<unsigned int>(v1.x);
            R.r14 = bitcast<float>(v1.y);
            R.r15 = bitcast<float>(v1.z);
            R.r16 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 48ull * cap)[idx];
            R.r17 = bitcast<float>(v2.x);
            R.r20 = bitcast<unsigned int>(v2.y);
            R.r21 = bitcast<unsigned int>(v2.z);
            R.r22 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 64ull * cap)[idx];
            R.r23 = bitcast<unsigned int>(v3.x);
            R.r24 = bitcast<unsigned int>(v3.y);
            R.r25 = bitcast<unsigned int>(v3.z);
            R.r130 = bitcast<unsigned int>(v3.w);
            const uint2 v4 = reinterpret_cast<const uint2*>(base + 80ull * cap)[idx];
            R.r131 = bitcast<unsigned int>(v4.x);
            return v4.y;
        }
        case 2: // bounce
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 88ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 104ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 120ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 136ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 152ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            return v4.w;
        }
        case 3: // isect
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 168ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 184ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 200ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 216ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 232ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 248ull * cap)[idx];
            R.r54 = bitcast<unsigned int>(v5.x);
            R.r55 = bitcast<unsigned int>(v5.y);
            R.r56 = bitcast<unsigned int>(v5.z);
            return v5.w;
        }
        case 4: // shade
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 264ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 280ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 296ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 312ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 328ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<float>(v4.w);
            const uint2 v5 = reinterpret_cast<const uint2*>(base + 344ull * cap)[idx];
            R.r54 = bitcast<unsigned int>(v5.x);
            return v5.y;
        }
        case 5: // hitp
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 352ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 368ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 384ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 400ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 416ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<float>(v4.w);
            const uint2 v5 = reinterpret_cast<const uint2*>(base + 432ull * cap)[idx];
            R.r54 = bitcast<unsigned int>(v5.x);
            return v5.y;
        }
        case 6: // emit
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 440ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r49 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 456ull * cap)[idx];
            R.r50 = bitcast<float>(v1.x);
            R.r51 = bitcast<float>(v1.y);
            R.r76 = bitcast<float>(v1.z);
            R.r77 = bitcast<float>(v1.w);
            const uint2 v2 = reinterpret_cast<const uint2*>(base + 472ull * cap)[idx];
            R.r78 = bitcast<float>(v2.x);
            return v2.y;
        }
        case 7: // surf
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 480ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 496ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 512ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 528ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 544ull * cap)[idx];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 560ull * cap)[idx];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 576ull * cap)[idx];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 8: // rrchk
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 592ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 608ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 624ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 640ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 656ull * cap)[idx];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 672ull * cap)[idx];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 688ull * cap)[idx];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 9: // rr_roll
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 704ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 720ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 736ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 752ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 768ull * cap)[idx];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 784ull * cap)[idx];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 800ull * cap)[idx];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 10: // rr
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 816ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 832ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 848ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 864ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 880ull * cap)[idx];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 896ull * cap)[idx];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 912ull * cap)[idx];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            R.r130 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 11: // rr_keep
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 928ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 944ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 960ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 976ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 992ull * cap)[idx];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1008ull * cap)[idx];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1024ull * cap)[idx];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            R.r86 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 12: // scatter
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1040ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1056ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1072ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1088ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1104ull * cap)[idx];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1120ull * cap)[idx];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1136ull * cap)[idx];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 13: // mirror
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1152ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1168ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1184ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1200ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1216ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1232ull * cap)[idx];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            return v5.w;
        }
        case 14: // diffuse
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1248ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1264ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1280ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1296ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1312ull * cap)[idx];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            return v4.w;
        }
        case 15: // disk_roll
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1328ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1344ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1360ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1376ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1392ull * cap)[idx];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            R.r100 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1408ull * cap)[idx];
            R.r101 = bitcast<float>(v5.x);
            R.r102 = bitcast<float>(v5.y);
            R.r103 = bitcast<float>(v5.z);
            R.r104 = bitcast<float>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(base + 1424ull * cap)[idx];
            R.r105 = bitcast<float>(v6.x);
            return v6.y;
        }
        case 16: // disk
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1432ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1448ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1464ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1480ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1496ull * cap)[idx];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            R.r100 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1512ull * cap)[idx];
            R.r101 = bitcast<float>(v5.x);
            R.r102 = bitcast<float>(v5.y);
            R.r103 = bitcast<float>(v5.z);
            R.r104 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1528ull * cap)[idx];
            R.r105 = bitcast<float>(v6.x);
            R.r130 = bitcast<unsigned int>(v6.y);
            R.r131 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 17: // disk_ok
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1544ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1560ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1576ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1592ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1608ull * cap)[idx];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            R.r100 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1624ull * cap)[idx];
            R.r101 = bitcast<float>(v5.x);
            R.r102 = bitcast<float>(v5.y);
            R.r103 = bitcast<float>(v5.z);
            R.r104 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1640ull * cap)[idx];
            R.r105 = bitcast<float>(v6.x);
            R.r106 = bitcast<float>(v6.y);
            R.r107 = bitcast<float>(v6.z);
            R.r108 = bitcast<float>(v6.w);
            const unsigned v7 = reinterpret_cast<const unsigned*>(base + 1656ull * cap)[idx];
            return v7;
        }
        case 18: // glass
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1664ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1680ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1696ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1712ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1728ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1744ull * cap)[idx];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r88 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1760ull * cap)[idx];
            R.r92 = bitcast<float>(v6.x);
            R.r93 = bitcast<float>(v6.y);
            R.r94 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 19: // refr
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1776ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1792ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1808ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1824ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1840ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1856ull * cap)[idx];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r88 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1872ull * cap)[idx];
            R.r111 = bitcast<float>(v6.x);
            R.r112 = bitcast<float>(v6.y);
            R.r113 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 20: // fres
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 1888ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 1904ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 1920ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 1936ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 1952ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 1968ull * cap)[idx];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r117 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 1984ull * cap)[idx];
            R.r118 = bitcast<float>(v6.x);
            R.r119 = bitcast<float>(v6.y);
            R.r127 = bitcast<float>(v6.z);
            R.r128 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2000ull * cap)[idx];
            R.r129 = bitcast<float>(v7.x);
            R.r130 = bitcast<unsigned int>(v7.y);
            return v7.z;
        }
        case 21: // take_refl
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2016ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2032ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2048ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2064ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2080ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2096ull * cap)[idx];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r128 = bitcast<float>(v5.w);
            const unsigned v6 = reinterpret_cast<const unsigned*>(base + 2112ull * cap)[idx];
            return v6;
        }
        case 22: // take_refr
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2120ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2136ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2152ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2168ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2184ull * cap)[idx];
            R.r117 = bitcast<float>(v4.x);
            R.r118 = bitcast<float>(v4.y);
            R.r119 = bitcast<float>(v4.z);
            R.r129 = bitcast<float>(v4.w);
            const unsigned v5 = reinterpret_cast<const unsigned*>(base + 2200ull * cap)[idx];
            return v5;
        }
        case 23: // roll
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2208ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r7 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2224ull * cap)[idx];
            R.r9 = bitcast<unsigned int>(v1.x);
            R.r11 = bitcast<unsigned int>(v1.y);
            R.r12 = bitcast<unsigned int>(v1.z);
            R.r13 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2240ull * cap)[idx];
            R.r14 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r16 = bitcast<float>(v2.z);
            R.r17 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2256ull * cap)[idx];
            R.r20 = bitcast<unsigned int>(v3.x);
            R.r21 = bitcast<unsigned int>(v3.y);
            R.r22 = bitcast<unsigned int>(v3.z);
            R.r23 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2272ull * cap)[idx];
            R.r24 = bitcast<unsigned int>(v4.x);
            R.r25 = bitcast<unsigned int>(v4.y);
            R.r26 = bitcast<unsigned int>(v4.z);
            R.r42 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2288ull * cap)[idx];
            R.r43 = bitcast<float>(v5.x);
            R.r44 = bitcast<float>(v5.y);
            R.r46 = bitcast<float>(v5.z);
            R.r47 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2304ull * cap)[idx];
            R.r48 = bitcast<float>(v6.x);
            R.r49 = bitcast<float>(v6.y);
            R.r50 = bitcast<float>(v6.z);
            R.r51 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(base + 2320ull * cap)[idx];
            R.r52 = bitcast<unsigned int>(v7.x);
            R.r76 = bitcast<float>(v7.y);
            R.r77 = bitcast<float>(v7.z);
            R.r78 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(base + 2336ull * cap)[idx];
            R.r79 = bitcast<unsigned int>(v8.x);
            R.r80 = bitcast<float>(v8.y);
            R.r81 = bitcast<float>(v8.z);
            R.r82 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(base + 2352ull * cap)[idx];
            R.r83 = bitcast<float>(v9.x);
            R.r84 = bitcast<float>(v9.y);
            R.r85 = bitcast<float>(v9.z);
            R.r87 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(base + 2368ull * cap)[idx];
            R.r92 = bitcast<float>(v10.x);
            R.r93 = bitcast<float>(v10.y);
            R.r94 = bitcast<float>(v10.z);
            R.r100 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(base + 2384ull * cap)[idx];
            R.r101 = bitcast<float>(v11.x);
            R.r102 = bitcast<float>(v11.y);
            R.r103 = bitcast<float>(v11.z);
            R.r104 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(base + 2400ull * cap)[idx];
            R.r105 = bitcast<float>(v12.x);
            R.r117 = bitcast<float>(v12.y);
            R.r118 = bitcast<float>(v12.z);
            R.r119 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(base + 2416ull * cap)[idx];
            R.r127 = bitcast<float>(v13.x);
            R.r128 = bitcast<float>(v13.y);
            R.r129 = bitcast<float>(v13.z);
            return v13.w;
        }
        case 24: // roll, context 0
        {
            R.r26 = static_cast<unsigned int>(0);
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2432ull * cap)[idx];
            R.r7 = bitcast<unsigned int>(v0.x);
            R.r9 = bitcast<unsigned int>(v0.y);
            R.r11 = bitcast<unsigned int>(v0.z);
            R.r12 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2448ull * cap)[idx];
            R.r13 = bitcast<unsigned int>(v1.x);
            R.r14 = bitcast<float>(v1.y);
            R.r15 = bitcast<float>(v1.z);
            R.r16 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2464ull * cap)[idx];
            R.r17 = bitcast<float>(v2.x);
            R.r20 = bitcast<unsigned int>(v2.y);
            R.r21 = bitcast<unsigned int>(v2.z);
            R.r22 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2480ull * cap)[idx];
            R.r23 = bitcast<unsigned int>(v3.x);
            R.r24 = bitcast<unsigned int>(v3.y);
            R.r25 = bitcast<unsigned int>(v3.z);
            return v3.w;
        }
        case 25: // roll, context 1
        {
            R.r26 = static_cast<unsigned int>(1);
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2496ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2512ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2528ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2544ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2560ull * cap)[idx];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2576ull * cap)[idx];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2592ull * cap)[idx];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 26: // roll, context 2
        {
            R.r26 = static_cast<unsigned int>(2);
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2608ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2624ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2640ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2656ull * cap)[idx];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2672ull * cap)[idx];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            R.r100 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2688ull * cap)[idx];
            R.r101 = bitcast<float>(v5.x);
            R.r102 = bitcast<float>(v5.y);
            R.r103 = bitcast<float>(v5.z);
            R.r104 = bitcast<float>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(base + 2704ull * cap)[idx];
            R.r105 = bitcast<float>(v6.x);
            return v6.y;
        }
        case 27: // roll, context 3
        {
            R.r26 = static_cast<unsigned int>(3);
            const uint4 v0 = reinterpret_cast<const uint4*>(base + 2712ull * cap)[idx];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(base + 2728ull * cap)[idx];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(base + 2744ull * cap)[idx];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(base + 2760ull * cap)[idx];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(base + 2776ull * cap)[idx];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(base + 2792ull * cap)[idx];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r117 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(base + 2808ull * cap)[idx];
            R.r118 = bitcast<float>(v6.x);
            R.r119 = bitcast<float>(v6.y);
            R.r127 = bitcast<float>(v6.z);
            R.r128 = bitcast<float>(v6.w);
            const uint2 v7 = reinterpret_cast<const uint2*>(base + 2824ull * cap)[idx];
            R.r129 = bitcast<float>(v7.x);
            return v7.y;
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
        case 0: bytes = 512u; break;
        case 1: bytes = 2304u; break;
        case 2: bytes = 2560u; break;
        case 3: bytes = 3072u; break;
        case 4: bytes = 2816u; break;
        case 5: bytes = 2816u; break;
        case 6: bytes = 1280u; break;
        case 7: bytes = 3584u; break;
        case 8: bytes = 3584u; break;
        case 9: bytes = 3584u; break;
        case 10: bytes = 3584u; break;
        case 11: bytes = 3584u; break;
        case 12: bytes = 3584u; break;
        case 13: bytes = 3072u; break;
        case 14: bytes = 2560u; break;
        case 15: bytes = 3328u; break;
        case 16: bytes = 3584u; break;
        case 17: bytes = 3712u; break;
        case 18: bytes = 3584u; break;
        case 19: bytes = 3584u; break;
        case 20: bytes = 4096u; break;
        case 21: bytes = 3200u; break;
        case 22: bytes = 2688u; break;
        case 23: bytes = 7168u; break;
        case 24: bytes = 2048u; break;
        case 25: bytes = 3584u; break;
        case 26: bytes = 3328u; break;
        case 27: bytes = 3840u; break;
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
            bulk_copy(stage + 1536u, base + 64ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 80ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 2:
            bulk_copy(stage + 0u, base + 88ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 3:
            bulk_copy(stage + 0u, base + 168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 4:
            bulk_copy(stage + 0u, base + 264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 344ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 5:
            bulk_copy(stage + 0u, base + 352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 432ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 6:
            bulk_copy(stage + 0u, base + 440ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 456ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 472ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 7:
            bulk_copy(stage + 0u, base + 480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 8:
            bulk_copy(stage + 0u, base + 592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 9:
            bulk_copy(stage + 0u, base + 704ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 720ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 736ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 752ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 768ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 784ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 800ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 10:
            bulk_copy(stage + 0u, base + 816ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 832ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 848ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 864ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 880ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 896ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 912ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 11:
            bulk_copy(stage + 0u, base + 928ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 944ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 960ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 976ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 992ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1008ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1024ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 12:
            bulk_copy(stage + 0u, base + 1040ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1056ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1072ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1088ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1104ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 13:
            bulk_copy(stage + 0u, base + 1152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1200ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1216ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1232ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 14:
            bulk_copy(stage + 0u, base + 1248ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1264ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1280ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1296ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1312ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 15:
            bulk_copy(stage + 0u, base + 1328ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1344ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1360ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1376ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1392ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1408ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1424ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 16:
            bulk_copy(stage + 0u, base + 1432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 17:
            bulk_copy(stage + 0u, base + 1544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 1656ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 18:
            bulk_copy(stage + 0u, base + 1664ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1680ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1696ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 19:
            bulk_copy(stage + 0u, base + 1776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1824ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1840ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1856ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1872ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 20:
            bulk_copy(stage + 0u, base + 1888ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 1904ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 1920ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 1936ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 1952ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 1968ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 1984ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2000ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 21:
            bulk_copy(stage + 0u, base + 2016ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2032ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2048ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2064ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2080ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2096ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2112ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 22:
            bulk_copy(stage + 0u, base + 2120ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2136ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2152ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2168ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2184ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2200ull * cap + static_cast<unsigned long long>(toff) * 4u, 128u, mbar);
            break;
        case 23:
            bulk_copy(stage + 0u, base + 2208ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2224ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2240ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2256ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2272ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2288ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2304ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2320ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4096u, base + 2336ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 4608u, base + 2352ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5120u, base + 2368ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 5632u, base + 2384ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6144u, base + 2400ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 6656u, base + 2416ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 24:
            bulk_copy(stage + 0u, base + 2432ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2448ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2464ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2480ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 25:
            bulk_copy(stage + 0u, base + 2496ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2512ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2528ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2544ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2560ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2576ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2592ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            break;
        case 26:
            bulk_copy(stage + 0u, base + 2608ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2624ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2640ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2656ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2672ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2688ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2704ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
            break;
        case 27:
            bulk_copy(stage + 0u, base + 2712ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 512u, base + 2728ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1024u, base + 2744ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 1536u, base + 2760ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2048u, base + 2776ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 2560u, base + 2792ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3072u, base + 2808ull * cap + static_cast<unsigned long long>(toff) * 16u, 512u, mbar);
            bulk_copy(stage + 3584u, base + 2824ull * cap + static_cast<unsigned long long>(toff) * 8u, 256u, mbar);
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
            R.r2 = bitcast<unsigned int>(v0.y);
            return v0.z;
        }
        case 1:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r7 = bitcast<unsigned int>(v0.x);
            R.r9 = bitcast<unsigned int>(v0.y);
            R.r11 = bitcast<unsigned int>(v0.z);
            R.r12 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r13 = bitcast<unsigned int>(v1.x);
            R.r14 = bitcast<float>(v1.y);
            R.r15 = bitcast<float>(v1.z);
            R.r16 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r17 = bitcast<float>(v2.x);
            R.r20 = bitcast<unsigned int>(v2.y);
            R.r21 = bitcast<unsigned int>(v2.z);
            R.r22 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r23 = bitcast<unsigned int>(v3.x);
            R.r24 = bitcast<unsigned int>(v3.y);
            R.r25 = bitcast<unsigned int>(v3.z);
            R.r130 = bitcast<unsigned int>(v3.w);
            const uint2 v4 = reinterpret_cast<const uint2*>(stage + 2048u)[lane];
            R.r131 = bitcast<unsigned int>(v4.x);
            return v4.y;
        }
        case 2:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            return v4.w;
        }
        case 3:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r54 = bitcast<unsigned int>(v5.x);
            R.r55 = bitcast<unsigned int>(v5.y);
            R.r56 = bitcast<unsigned int>(v5.z);
            return v5.w;
        }
        case 4:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<float>(v4.w);
            const uint2 v5 = reinterpret_cast<const uint2*>(stage + 2560u)[lane];
            R.r54 = bitcast<unsigned int>(v5.x);
            return v5.y;
        }
        case 5:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r53 = bitcast<float>(v4.w);
            const uint2 v5 = reinterpret_cast<const uint2*>(stage + 2560u)[lane];
            R.r54 = bitcast<unsigned int>(v5.x);
            return v5.y;
        }
        case 6:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r49 = bitcast<float>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r50 = bitcast<float>(v1.x);
            R.r51 = bitcast<float>(v1.y);
            R.r76 = bitcast<float>(v1.z);
            R.r77 = bitcast<float>(v1.w);
            const uint2 v2 = reinterpret_cast<const uint2*>(stage + 1024u)[lane];
            R.r78 = bitcast<float>(v2.x);
            return v2.y;
        }
        case 7:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 8:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 9:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 10:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            R.r130 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 11:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            R.r86 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 12:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 13:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            return v5.w;
        }
        case 14:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            return v4.w;
        }
        case 15:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            R.r100 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r101 = bitcast<float>(v5.x);
            R.r102 = bitcast<float>(v5.y);
            R.r103 = bitcast<float>(v5.z);
            R.r104 = bitcast<float>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(stage + 3072u)[lane];
            R.r105 = bitcast<float>(v6.x);
            return v6.y;
        }
        case 16:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            R.r100 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r101 = bitcast<float>(v5.x);
            R.r102 = bitcast<float>(v5.y);
            R.r103 = bitcast<float>(v5.z);
            R.r104 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r105 = bitcast<float>(v6.x);
            R.r130 = bitcast<unsigned int>(v6.y);
            R.r131 = bitcast<unsigned int>(v6.z);
            return v6.w;
        }
        case 17:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            R.r100 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r101 = bitcast<float>(v5.x);
            R.r102 = bitcast<float>(v5.y);
            R.r103 = bitcast<float>(v5.z);
            R.r104 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r105 = bitcast<float>(v6.x);
            R.r106 = bitcast<float>(v6.y);
            R.r107 = bitcast<float>(v6.z);
            R.r108 = bitcast<float>(v6.w);
            const unsigned v7 = reinterpret_cast<const unsigned*>(stage + 3584u)[lane];
            return v7;
        }
        case 18:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r88 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r92 = bitcast<float>(v6.x);
            R.r93 = bitcast<float>(v6.y);
            R.r94 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 19:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r88 = bitcast<unsigned int>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r111 = bitcast<float>(v6.x);
            R.r112 = bitcast<float>(v6.y);
            R.r113 = bitcast<float>(v6.z);
            return v6.w;
        }
        case 20:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r117 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r118 = bitcast<float>(v6.x);
            R.r119 = bitcast<float>(v6.y);
            R.r127 = bitcast<float>(v6.z);
            R.r128 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r129 = bitcast<float>(v7.x);
            R.r130 = bitcast<unsigned int>(v7.y);
            return v7.z;
        }
        case 21:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r128 = bitcast<float>(v5.w);
            const unsigned v6 = reinterpret_cast<const unsigned*>(stage + 3072u)[lane];
            return v6;
        }
        case 22:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r117 = bitcast<float>(v4.x);
            R.r118 = bitcast<float>(v4.y);
            R.r119 = bitcast<float>(v4.z);
            R.r129 = bitcast<float>(v4.w);
            const unsigned v5 = reinterpret_cast<const unsigned*>(stage + 2560u)[lane];
            return v5;
        }
        case 23:
        {
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r7 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r9 = bitcast<unsigned int>(v1.x);
            R.r11 = bitcast<unsigned int>(v1.y);
            R.r12 = bitcast<unsigned int>(v1.z);
            R.r13 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r14 = bitcast<float>(v2.x);
            R.r15 = bitcast<float>(v2.y);
            R.r16 = bitcast<float>(v2.z);
            R.r17 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r20 = bitcast<unsigned int>(v3.x);
            R.r21 = bitcast<unsigned int>(v3.y);
            R.r22 = bitcast<unsigned int>(v3.z);
            R.r23 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r24 = bitcast<unsigned int>(v4.x);
            R.r25 = bitcast<unsigned int>(v4.y);
            R.r26 = bitcast<unsigned int>(v4.z);
            R.r42 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r43 = bitcast<float>(v5.x);
            R.r44 = bitcast<float>(v5.y);
            R.r46 = bitcast<float>(v5.z);
            R.r47 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r48 = bitcast<float>(v6.x);
            R.r49 = bitcast<float>(v6.y);
            R.r50 = bitcast<float>(v6.z);
            R.r51 = bitcast<float>(v6.w);
            const uint4 v7 = reinterpret_cast<const uint4*>(stage + 3584u)[lane];
            R.r52 = bitcast<unsigned int>(v7.x);
            R.r76 = bitcast<float>(v7.y);
            R.r77 = bitcast<float>(v7.z);
            R.r78 = bitcast<float>(v7.w);
            const uint4 v8 = reinterpret_cast<const uint4*>(stage + 4096u)[lane];
            R.r79 = bitcast<unsigned int>(v8.x);
            R.r80 = bitcast<float>(v8.y);
            R.r81 = bitcast<float>(v8.z);
            R.r82 = bitcast<float>(v8.w);
            const uint4 v9 = reinterpret_cast<const uint4*>(stage + 4608u)[lane];
            R.r83 = bitcast<float>(v9.x);
            R.r84 = bitcast<float>(v9.y);
            R.r85 = bitcast<float>(v9.z);
            R.r87 = bitcast<float>(v9.w);
            const uint4 v10 = reinterpret_cast<const uint4*>(stage + 5120u)[lane];
            R.r92 = bitcast<float>(v10.x);
            R.r93 = bitcast<float>(v10.y);
            R.r94 = bitcast<float>(v10.z);
            R.r100 = bitcast<float>(v10.w);
            const uint4 v11 = reinterpret_cast<const uint4*>(stage + 5632u)[lane];
            R.r101 = bitcast<float>(v11.x);
            R.r102 = bitcast<float>(v11.y);
            R.r103 = bitcast<float>(v11.z);
            R.r104 = bitcast<float>(v11.w);
            const uint4 v12 = reinterpret_cast<const uint4*>(stage + 6144u)[lane];
            R.r105 = bitcast<float>(v12.x);
            R.r117 = bitcast<float>(v12.y);
            R.r118 = bitcast<float>(v12.z);
            R.r119 = bitcast<float>(v12.w);
            const uint4 v13 = reinterpret_cast<const uint4*>(stage + 6656u)[lane];
            R.r127 = bitcast<float>(v13.x);
            R.r128 = bitcast<float>(v13.y);
            R.r129 = bitcast<float>(v13.z);
            return v13.w;
        }
        case 24:
        {
            R.r26 = static_cast<unsigned int>(0);
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r7 = bitcast<unsigned int>(v0.x);
            R.r9 = bitcast<unsigned int>(v0.y);
            R.r11 = bitcast<unsigned int>(v0.z);
            R.r12 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r13 = bitcast<unsigned int>(v1.x);
            R.r14 = bitcast<float>(v1.y);
            R.r15 = bitcast<float>(v1.z);
            R.r16 = bitcast<float>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r17 = bitcast<float>(v2.x);
            R.r20 = bitcast<unsigned int>(v2.y);
            R.r21 = bitcast<unsigned int>(v2.z);
            R.r22 = bitcast<unsigned int>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r23 = bitcast<unsigned int>(v3.x);
            R.r24 = bitcast<unsigned int>(v3.y);
            R.r25 = bitcast<unsigned int>(v3.z);
            return v3.w;
        }
        case 25:
        {
            R.r26 = static_cast<unsigned int>(1);
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r76 = bitcast<float>(v4.x);
            R.r77 = bitcast<float>(v4.y);
            R.r78 = bitcast<float>(v4.z);
            R.r79 = bitcast<unsigned int>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r80 = bitcast<float>(v5.x);
            R.r81 = bitcast<float>(v5.y);
            R.r82 = bitcast<float>(v5.z);
            R.r83 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r84 = bitcast<float>(v6.x);
            R.r85 = bitcast<float>(v6.y);
            return v6.z;
        }
        case 26:
        {
            R.r26 = static_cast<unsigned int>(2);
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r46 = bitcast<float>(v2.y);
            R.r47 = bitcast<float>(v2.z);
            R.r48 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r49 = bitcast<float>(v3.x);
            R.r50 = bitcast<float>(v3.y);
            R.r51 = bitcast<float>(v3.z);
            R.r52 = bitcast<unsigned int>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r92 = bitcast<float>(v4.x);
            R.r93 = bitcast<float>(v4.y);
            R.r94 = bitcast<float>(v4.z);
            R.r100 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r101 = bitcast<float>(v5.x);
            R.r102 = bitcast<float>(v5.y);
            R.r103 = bitcast<float>(v5.z);
            R.r104 = bitcast<float>(v5.w);
            const uint2 v6 = reinterpret_cast<const uint2*>(stage + 3072u)[lane];
            R.r105 = bitcast<float>(v6.x);
            return v6.y;
        }
        case 27:
        {
            R.r26 = static_cast<unsigned int>(3);
            const uint4 v0 = reinterpret_cast<const uint4*>(stage + 0u)[lane];
            R.r3 = bitcast<float>(v0.x);
            R.r4 = bitcast<float>(v0.y);
            R.r5 = bitcast<float>(v0.z);
            R.r11 = bitcast<unsigned int>(v0.w);
            const uint4 v1 = reinterpret_cast<const uint4*>(stage + 512u)[lane];
            R.r12 = bitcast<unsigned int>(v1.x);
            R.r13 = bitcast<unsigned int>(v1.y);
            R.r23 = bitcast<unsigned int>(v1.z);
            R.r24 = bitcast<unsigned int>(v1.w);
            const uint4 v2 = reinterpret_cast<const uint4*>(stage + 1024u)[lane];
            R.r25 = bitcast<unsigned int>(v2.x);
            R.r42 = bitcast<float>(v2.y);
            R.r43 = bitcast<float>(v2.z);
            R.r44 = bitcast<float>(v2.w);
            const uint4 v3 = reinterpret_cast<const uint4*>(stage + 1536u)[lane];
            R.r46 = bitcast<float>(v3.x);
            R.r47 = bitcast<float>(v3.y);
            R.r48 = bitcast<float>(v3.z);
            R.r49 = bitcast<float>(v3.w);
            const uint4 v4 = reinterpret_cast<const uint4*>(stage + 2048u)[lane];
            R.r50 = bitcast<float>(v4.x);
            R.r51 = bitcast<float>(v4.y);
            R.r52 = bitcast<unsigned int>(v4.z);
            R.r83 = bitcast<float>(v4.w);
            const uint4 v5 = reinterpret_cast<const uint4*>(stage + 2560u)[lane];
            R.r84 = bitcast<float>(v5.x);
            R.r85 = bitcast<float>(v5.y);
            R.r87 = bitcast<float>(v5.z);
            R.r117 = bitcast<float>(v5.w);
            const uint4 v6 = reinterpret_cast<const uint4*>(stage + 3072u)[lane];
            R.r118 = bitcast<float>(v6.x);
            R.r119 = bitcast<float>(v6.y);
            R.r127 = bitcast<float>(v6.z);
            R.r128 = bitcast<float>(v6.w);
            const uint2 v7 = reinterpret_cast<const uint2*>(stage + 3584u)[lane];
            R.r129 = bitcast<float>(v7.x);
            return v7.y;
        }
        default: return 0xffffffffu;
        }
    }
};

const int kInTypes[] = {LOOM_B200_U32, LOOM_B200_U32};
const int kOutTypes[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kInNames[] = {"inst", "sid"};
const char* const kOutNames[] = {"L0", "L1", "L2"};
const uint32_t kInstrs[] = {32, 63, 5, 38, 2, 28, 4, 3, 2, 2, 4, 4, 18, 5, 26, 2, 8, 20, 13, 40, 2, 4, 7, 292};
const uint32_t kLive[] = {164, 132, 176, 192, 184, 184, 36, 216, 216, 216, 192, 192, 188, 188, 192, 216, 224, 176, 220, 208, 192, 188, 164, 220};

const loom_b200_kernel_info kInfo = {
    "sphere_pt_f32", "144eab9a4253b9da", 2u, 3u, kInTypes, kOutTypes, kInNames, kOutNames,
    24u, 134u, 536u, 71u, kInstrs, kLive};

const uint32_t kQRegs0[] = {1u, 2u};
const int kQTypes0[] = {LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames0[] = {"inst", "sid"};
const unsigned long long kQOffs0[] = {0ull, 0ull};
const unsigned kQSubs0[] = {0u, 4u};
const unsigned kQWidths0[] = {16u, 16u};
const uint32_t kQRegs1[] = {7u, 9u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 20u, 21u, 22u, 23u, 24u, 25u, 130u, 131u};
const int kQTypes1[] = {LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames1[] = {"w", "h", "k0", "soff", "scnt", "cam0", "cam1", "cam2", "tanf", "smp", "px", "py", "k2", "c0", "c1", "u0", "u1"};
const unsigned long long kQOffs1[] = {16ull, 16ull, 16ull, 16ull, 32ull, 32ull, 32ull, 32ull, 48ull, 48ull, 48ull, 48ull, 64ull, 64ull, 64ull, 64ull, 80ull};
const unsigned kQSubs1[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths1[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs2[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u};
const int kQTypes2[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames2[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth"};
const unsigned long long kQOffs2[] = {88ull, 88ull, 88ull, 88ull, 104ull, 104ull, 104ull, 104ull, 120ull, 120ull, 120ull, 120ull, 136ull, 136ull, 136ull, 136ull, 152ull, 152ull, 152ull};
const unsigned kQSubs2[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths2[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs3[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 53u, 54u, 55u, 56u};
const int kQTypes3[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames3[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "tmin", "hid", "i", "sp"};
const unsigned long long kQOffs3[] = {168ull, 168ull, 168ull, 168ull, 184ull, 184ull, 184ull, 184ull, 200ull, 200ull, 200ull, 200ull, 216ull, 216ull, 216ull, 216ull, 232ull, 232ull, 232ull, 232ull, 248ull, 248ull, 248ull};
const unsigned kQSubs3[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths3[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs4[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 53u, 54u};
const int kQTypes4[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames4[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "tmin", "hid"};
const unsigned long long kQOffs4[] = {264ull, 264ull, 264ull, 264ull, 280ull, 280ull, 280ull, 280ull, 296ull, 296ull, 296ull, 296ull, 312ull, 312ull, 312ull, 312ull, 328ull, 328ull, 328ull, 328ull, 344ull};
const unsigned kQSubs4[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths4[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs5[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 53u, 54u};
const int kQTypes5[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames5[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "tmin", "hid"};
const unsigned long long kQOffs5[] = {352ull, 352ull, 352ull, 352ull, 368ull, 368ull, 368ull, 368ull, 384ull, 384ull, 384ull, 384ull, 400ull, 400ull, 400ull, 400ull, 416ull, 416ull, 416ull, 416ull, 432ull};
const unsigned kQSubs5[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths5[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs6[] = {3u, 4u, 5u, 49u, 50u, 51u, 76u, 77u, 78u};
const int kQTypes6[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames6[] = {"L0", "L1", "L2", "T0", "T1", "T2", "cr", "cg", "cb"};
const unsigned long long kQOffs6[] = {440ull, 440ull, 440ull, 440ull, 456ull, 456ull, 456ull, 456ull, 472ull};
const unsigned kQSubs6[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths6[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs7[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes7[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames7[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs7[] = {480ull, 480ull, 480ull, 480ull, 496ull, 496ull, 496ull, 496ull, 512ull, 512ull, 512ull, 512ull, 528ull, 528ull, 528ull, 528ull, 544ull, 544ull, 544ull, 544ull, 560ull, 560ull, 560ull, 560ull, 576ull, 576ull};
const unsigned kQSubs7[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths7[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs8[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes8[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames8[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs8[] = {592ull, 592ull, 592ull, 592ull, 608ull, 608ull, 608ull, 608ull, 624ull, 624ull, 624ull, 624ull, 640ull, 640ull, 640ull, 640ull, 656ull, 656ull, 656ull, 656ull, 672ull, 672ull, 672ull, 672ull, 688ull, 688ull};
const unsigned kQSubs8[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths8[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs9[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes9[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames9[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs9[] = {704ull, 704ull, 704ull, 704ull, 720ull, 720ull, 720ull, 720ull, 736ull, 736ull, 736ull, 736ull, 752ull, 752ull, 752ull, 752ull, 768ull, 768ull, 768ull, 768ull, 784ull, 784ull, 784ull, 784ull, 800ull, 800ull};
const unsigned kQSubs9[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths9[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs10[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u, 130u};
const int kQTypes10[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames10[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2", "u0"};
const unsigned long long kQOffs10[] = {816ull, 816ull, 816ull, 816ull, 832ull, 832ull, 832ull, 832ull, 848ull, 848ull, 848ull, 848ull, 864ull, 864ull, 864ull, 864ull, 880ull, 880ull, 880ull, 880ull, 896ull, 896ull, 896ull, 896ull, 912ull, 912ull, 912ull};
const unsigned kQSubs10[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths10[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs11[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u, 86u};
const int kQTypes11[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames11[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2", "p"};
const unsigned long long kQOffs11[] = {928ull, 928ull, 928ull, 928ull, 944ull, 944ull, 944ull, 944ull, 960ull, 960ull, 960ull, 960ull, 976ull, 976ull, 976ull, 976ull, 992ull, 992ull, 992ull, 992ull, 1008ull, 1008ull, 1008ull, 1008ull, 1024ull, 1024ull, 1024ull};
const unsigned kQSubs11[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths11[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs12[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes12[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames12[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs12[] = {1040ull, 1040ull, 1040ull, 1040ull, 1056ull, 1056ull, 1056ull, 1056ull, 1072ull, 1072ull, 1072ull, 1072ull, 1088ull, 1088ull, 1088ull, 1088ull, 1104ull, 1104ull, 1104ull, 1104ull, 1120ull, 1120ull, 1120ull, 1120ull, 1136ull, 1136ull};
const unsigned kQSubs12[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths12[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs13[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u};
const int kQTypes13[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames13[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn"};
const unsigned long long kQOffs13[] = {1152ull, 1152ull, 1152ull, 1152ull, 1168ull, 1168ull, 1168ull, 1168ull, 1184ull, 1184ull, 1184ull, 1184ull, 1200ull, 1200ull, 1200ull, 1200ull, 1216ull, 1216ull, 1216ull, 1216ull, 1232ull, 1232ull, 1232ull};
const unsigned kQSubs13[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths13[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs14[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u};
const int kQTypes14[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames14[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2"};
const unsigned long long kQOffs14[] = {1248ull, 1248ull, 1248ull, 1248ull, 1264ull, 1264ull, 1264ull, 1264ull, 1280ull, 1280ull, 1280ull, 1280ull, 1296ull, 1296ull, 1296ull, 1296ull, 1312ull, 1312ull, 1312ull};
const unsigned kQSubs14[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths14[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs15[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u};
const int kQTypes15[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames15[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2"};
const unsigned long long kQOffs15[] = {1328ull, 1328ull, 1328ull, 1328ull, 1344ull, 1344ull, 1344ull, 1344ull, 1360ull, 1360ull, 1360ull, 1360ull, 1376ull, 1376ull, 1376ull, 1376ull, 1392ull, 1392ull, 1392ull, 1392ull, 1408ull, 1408ull, 1408ull, 1408ull, 1424ull};
const unsigned kQSubs15[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths15[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs16[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u, 130u, 131u};
const int kQTypes16[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames16[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2", "u0", "u1"};
const unsigned long long kQOffs16[] = {1432ull, 1432ull, 1432ull, 1432ull, 1448ull, 1448ull, 1448ull, 1448ull, 1464ull, 1464ull, 1464ull, 1464ull, 1480ull, 1480ull, 1480ull, 1480ull, 1496ull, 1496ull, 1496ull, 1496ull, 1512ull, 1512ull, 1512ull, 1512ull, 1528ull, 1528ull, 1528ull};
const unsigned kQSubs16[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths16[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs17[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u, 106u, 107u, 108u};
const int kQTypes17[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames17[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2", "dx", "dy", "rr2"};
const unsigned long long kQOffs17[] = {1544ull, 1544ull, 1544ull, 1544ull, 1560ull, 1560ull, 1560ull, 1560ull, 1576ull, 1576ull, 1576ull, 1576ull, 1592ull, 1592ull, 1592ull, 1592ull, 1608ull, 1608ull, 1608ull, 1608ull, 1624ull, 1624ull, 1624ull, 1624ull, 1640ull, 1640ull, 1640ull, 1640ull};
const unsigned kQSubs17[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths17[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs18[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 88u, 92u, 93u, 94u};
const int kQTypes18[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames18[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "into", "nl0", "nl1", "nl2"};
const unsigned long long kQOffs18[] = {1664ull, 1664ull, 1664ull, 1664ull, 1680ull, 1680ull, 1680ull, 1680ull, 1696ull, 1696ull, 1696ull, 1696ull, 1712ull, 1712ull, 1712ull, 1712ull, 1728ull, 1728ull, 1728ull, 1728ull, 1744ull, 1744ull, 1744ull, 1744ull, 1760ull, 1760ull, 1760ull};
const unsigned kQSubs18[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths18[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs19[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 88u, 111u, 112u, 113u};
const int kQTypes19[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames19[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "into", "nnt", "ddn", "c2"};
const unsigned long long kQOffs19[] = {1776ull, 1776ull, 1776ull, 1776ull, 1792ull, 1792ull, 1792ull, 1792ull, 1808ull, 1808ull, 1808ull, 1808ull, 1824ull, 1824ull, 1824ull, 1824ull, 1840ull, 1840ull, 1840ull, 1840ull, 1856ull, 1856ull, 1856ull, 1856ull, 1872ull, 1872ull, 1872ull};
const unsigned kQSubs19[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths19[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs20[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 117u, 118u, 119u, 127u, 128u, 129u, 130u};
const int kQTypes20[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames20[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "td0", "td1", "td2", "pp", "rp", "tp", "u0"};
const unsigned long long kQOffs20[] = {1888ull, 1888ull, 1888ull, 1888ull, 1904ull, 1904ull, 1904ull, 1904ull, 1920ull, 1920ull, 1920ull, 1920ull, 1936ull, 1936ull, 1936ull, 1936ull, 1952ull, 1952ull, 1952ull, 1952ull, 1968ull, 1968ull, 1968ull, 1968ull, 1984ull, 1984ull, 1984ull, 1984ull, 2000ull, 2000ull};
const unsigned kQSubs20[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths20[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs21[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 128u};
const int kQTypes21[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames21[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "rp"};
const unsigned long long kQOffs21[] = {2016ull, 2016ull, 2016ull, 2016ull, 2032ull, 2032ull, 2032ull, 2032ull, 2048ull, 2048ull, 2048ull, 2048ull, 2064ull, 2064ull, 2064ull, 2064ull, 2080ull, 2080ull, 2080ull, 2080ull, 2096ull, 2096ull, 2096ull, 2096ull};
const unsigned kQSubs21[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths21[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs22[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 117u, 118u, 119u, 129u};
const int kQTypes22[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames22[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "td0", "td1", "td2", "tp"};
const unsigned long long kQOffs22[] = {2120ull, 2120ull, 2120ull, 2120ull, 2136ull, 2136ull, 2136ull, 2136ull, 2152ull, 2152ull, 2152ull, 2152ull, 2168ull, 2168ull, 2168ull, 2168ull, 2184ull, 2184ull, 2184ull, 2184ull};
const unsigned kQSubs22[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u};
const unsigned kQWidths22[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs23[] = {3u, 4u, 5u, 7u, 9u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 20u, 21u, 22u, 23u, 24u, 25u, 26u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u, 87u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u, 117u, 118u, 119u, 127u, 128u, 129u};
const int kQTypes23[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames23[] = {"L0", "L1", "L2", "w", "h", "k0", "soff", "scnt", "cam0", "cam1", "cam2", "tanf", "smp", "px", "py", "k2", "c0", "c1", "rpt", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2", "dn", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2", "td0", "td1", "td2", "pp", "rp", "tp"};
const unsigned long long kQOffs23[] = {2208ull, 2208ull, 2208ull, 2208ull, 2224ull, 2224ull, 2224ull, 2224ull, 2240ull, 2240ull, 2240ull, 2240ull, 2256ull, 2256ull, 2256ull, 2256ull, 2272ull, 2272ull, 2272ull, 2272ull, 2288ull, 2288ull, 2288ull, 2288ull, 2304ull, 2304ull, 2304ull, 2304ull, 2320ull, 2320ull, 2320ull, 2320ull, 2336ull, 2336ull, 2336ull, 2336ull, 2352ull, 2352ull, 2352ull, 2352ull, 2368ull, 2368ull, 2368ull, 2368ull, 2384ull, 2384ull, 2384ull, 2384ull, 2400ull, 2400ull, 2400ull, 2400ull, 2416ull, 2416ull, 2416ull};
const unsigned kQSubs23[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths23[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs24[] = {7u, 9u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 20u, 21u, 22u, 23u, 24u, 25u};
const int kQTypes24[] = {LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames24[] = {"w", "h", "k0", "soff", "scnt", "cam0", "cam1", "cam2", "tanf", "smp", "px", "py", "k2", "c0", "c1"};
const unsigned long long kQOffs24[] = {2432ull, 2432ull, 2432ull, 2432ull, 2448ull, 2448ull, 2448ull, 2448ull, 2464ull, 2464ull, 2464ull, 2464ull, 2480ull, 2480ull, 2480ull};
const unsigned kQSubs24[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u};
const unsigned kQWidths24[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs25[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes25[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames25[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs25[] = {2496ull, 2496ull, 2496ull, 2496ull, 2512ull, 2512ull, 2512ull, 2512ull, 2528ull, 2528ull, 2528ull, 2528ull, 2544ull, 2544ull, 2544ull, 2544ull, 2560ull, 2560ull, 2560ull, 2560ull, 2576ull, 2576ull, 2576ull, 2576ull, 2592ull, 2592ull};
const unsigned kQSubs25[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u};
const unsigned kQWidths25[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u};
const uint32_t kQRegs26[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u};
const int kQTypes26[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames26[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2"};
const unsigned long long kQOffs26[] = {2608ull, 2608ull, 2608ull, 2608ull, 2624ull, 2624ull, 2624ull, 2624ull, 2640ull, 2640ull, 2640ull, 2640ull, 2656ull, 2656ull, 2656ull, 2656ull, 2672ull, 2672ull, 2672ull, 2672ull, 2688ull, 2688ull, 2688ull, 2688ull, 2704ull};
const unsigned kQSubs26[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths26[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const uint32_t kQRegs27[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 117u, 118u, 119u, 127u, 128u, 129u};
const int kQTypes27[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames27[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "td0", "td1", "td2", "pp", "rp", "tp"};
const unsigned long long kQOffs27[] = {2712ull, 2712ull, 2712ull, 2712ull, 2728ull, 2728ull, 2728ull, 2728ull, 2744ull, 2744ull, 2744ull, 2744ull, 2760ull, 2760ull, 2760ull, 2760ull, 2776ull, 2776ull, 2776ull, 2776ull, 2792ull, 2792ull, 2792ull, 2792ull, 2808ull, 2808ull, 2808ull, 2808ull, 2824ull};
const unsigned kQSubs27[] = {0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u, 4u, 8u, 12u, 0u};
const unsigned kQWidths27[] = {16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 16u, 8u};
const loom_b200_queue_layout kQueues[] = {
    {0u, -1, 2u, kQRegs0, kQTypes0, kQNames0},
    {1u, -1, 17u, kQRegs1, kQTypes1, kQNames1},
    {2u, -1, 19u, kQRegs2, kQTypes2, kQNames2},
    {3u, -1, 23u, kQRegs3, kQTypes3, kQNames3},
    {4u, -1, 21u, kQRegs4, kQTypes4, kQNames4},
    {5u, -1, 21u, kQRegs5, kQTypes5, kQNames5},
    {6u, -1, 9u, kQRegs6, kQTypes6, kQNames6},
    {7u, -1, 26u, kQRegs7, kQTypes7, kQNames7},
    {8u, -1, 26u, kQRegs8, kQTypes8, kQNames8},
    {9u, -1, 26u, kQRegs9, kQTypes9, kQNames9},
    {10u, -1, 27u, kQRegs10, kQTypes10, kQNames10},
    {11u, -1, 27u, kQRegs11, kQTypes11, kQNames11},
    {12u, -1, 26u, kQRegs12, kQTypes12, kQNames12},
    {13u, -1, 23u, kQRegs13, kQTypes13, kQNames13},
    {14u, -1, 19u, kQRegs14, kQTypes14, kQNames14},
    {15u, -1, 25u, kQRegs15, kQTypes15, kQNames15},
    {16u, -1, 27u, kQRegs16, kQTypes16, kQNames16},
    {17u, -1, 28u, kQRegs17, kQTypes17, kQNames17},
    {18u, -1, 27u, kQRegs18, kQTypes18, kQNames18},
    {19u, -1, 27u, kQRegs19, kQTypes19, kQNames19},
    {20u, -1, 30u, kQRegs20, kQTypes20, kQNames20},
    {21u, -1, 24u, kQRegs21, kQTypes21, kQNames21},
    {22u, -1, 20u, kQRegs22, kQTypes22, kQNames22},
    {23u, -1, 55u, kQRegs23, kQTypes23, kQNames23},
    {23u, 0, 15u, kQRegs24, kQTypes24, kQNames24},
    {23u, 1, 26u, kQRegs25, kQTypes25, kQNames25},
    {23u, 2, 25u, kQRegs26, kQTypes26, kQNames26},
    {23u, 3, 29u, kQRegs27, kQTypes27, kQNames27},
};
const QueueSegment kSegments[] = {
    {kQOffs0, kQSubs0, kQWidths0, 0ull, 8u, 16u},
    {kQOffs1, kQSubs1, kQWidths1, 80ull, 4u, 8u},
    {kQOffs2, kQSubs2, kQWidths2, 152ull, 12u, 16u},
    {kQOffs3, kQSubs3, kQWidths3, 248ull, 12u, 16u},
    {kQOffs4, kQSubs4, kQWidths4, 344ull, 4u, 8u},
    {kQOffs5, kQSubs5, kQWidths5, 432ull, 4u, 8u},
    {kQOffs6, kQSubs6, kQWidths6, 472ull, 4u, 8u},
    {kQOffs7, kQSubs7, kQWidths7, 576ull, 8u, 16u},
    {kQOffs8, kQSubs8, kQWidths8, 688ull, 8u, 16u},
    {kQOffs9, kQSubs9, kQWidths9, 800ull, 8u, 16u},
    {kQOffs10, kQSubs10, kQWidths10, 912ull, 12u, 16u},
    {kQOffs11, kQSubs11, kQWidths11, 1024ull, 12u, 16u},
    {kQOffs12, kQSubs12, kQWidths12, 1136ull, 8u, 16u},
    {kQOffs13, kQSubs13, kQWidths13, 1232ull, 12u, 16u},
    {kQOffs14, kQSubs14, kQWidths14, 1312ull, 12u, 16u},
    {kQOffs15, kQSubs15, kQWidths15, 1424ull, 4u, 8u},
    {kQOffs16, kQSubs16, kQWidths16, 1528ull, 12u, 16u},
    {kQOffs17, kQSubs17, kQWidths17, 1656ull, 0u, 4u},
    {kQOffs18, kQSubs18, kQWidths18, 1760ull, 12u, 16u},
    {kQOffs19, kQSubs19, kQWidths19, 1872ull, 12u, 16u},
    {kQOffs20, kQSubs20, kQWidths20, 2000ull, 8u, 16u},
    {kQOffs21, kQSubs21, kQWidths21, 2112ull, 0u, 4u},
    {kQOffs22, kQSubs22, kQWidths22, 2200ull, 0u, 4u},
    {kQOffs23, kQSubs23, kQWidths23, 2416ull, 12u, 16u},
    {kQOffs24, kQSubs24, kQWidths24, 2480ull, 12u, 16u},
    {kQOffs25, kQSubs25, kQWidths25, 2592ull, 8u, 16u},
    {kQOffs26, kQSubs26, kQWidths26, 2704ull, 4u, 8u},
    {kQOffs27, kQSubs27, kQWidths27, 2824ull, 4u, 8u},
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

} } // namespace loom_b200::k_sphere_pt_f32

extern const loom_b200::KernelEntry loom_b200_entry_sphere_pt_f32;
const loom_b200::KernelEntry loom_b200_entry_sphere_pt_f32 = {
    &loom_b200::k_sphere_pt_f32::kInfo, loom_b200::k_sphere_pt_f32::K::kRowBytes, 28,
    &loom_b200::k_sphere_pt_f32::launch_plain, &loom_b200::k_sphere_pt_f32::launch_regroup,
    &loom_b200::k_sphere_pt_f32::regroup_occupancy,
    loom_b200::k_sphere_pt_f32::kQueues, loom_b200::k_sphere_pt_f32::kSegments,
    loom_b200::k_sphere_pt_f32::kRegCaps, 8u, loom_b200::k_sphere_pt_f32::K::kMaxStageRow};
