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
            reinterpret_cast<unsigned int*>(base + 0ull * cap)[idx] = R.r1;
            reinterpret_cast<unsigned int*>(base + 4ull * cap)[idx] = R.r2;
            reinterpret_cast<unsigned*>(base + 8ull * cap)[idx] = tid;
            return;
        case 1: // prim
            reinterpret_cast<unsigned int*>(base + 16ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 20ull * cap)[idx] = R.r9;
            reinterpret_cast<unsigned int*>(base + 24ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 28ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 32ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 36ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 40ull * cap)[idx] = R.r15;
            reinterpret_cast<float*>(base + 44ull * cap)[idx] = R.r16;
            reinterpret_cast<float*>(base + 48ull * cap)[idx] = R.r17;
            reinterpret_cast<unsigned int*>(base + 52ull * cap)[idx] = R.r20;
            reinterpret_cast<unsigned int*>(base + 56ull * cap)[idx] = R.r21;
            reinterpret_cast<unsigned int*>(base + 60ull * cap)[idx] = R.r22;
            reinterpret_cast<unsigned int*>(base + 64ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 68ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 72ull * cap)[idx] = R.r25;
            reinterpret_cast<unsigned int*>(base + 76ull * cap)[idx] = R.r130;
            reinterpret_cast<unsigned int*>(base + 80ull * cap)[idx] = R.r131;
            reinterpret_cast<unsigned*>(base + 84ull * cap)[idx] = tid;
            return;
        case 2: // bounce
            reinterpret_cast<float*>(base + 88ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 92ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 96ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 100ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 104ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 108ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 112ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 116ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 120ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 124ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 128ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 132ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 136ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 140ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 144ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 148ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 152ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 156ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 160ull * cap)[idx] = R.r52;
            reinterpret_cast<unsigned*>(base + 164ull * cap)[idx] = tid;
            return;
        case 3: // isect
            reinterpret_cast<float*>(base + 168ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 172ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 176ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 180ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 184ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 188ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 192ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 196ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 200ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 204ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 208ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 212ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 216ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 220ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 224ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 228ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 232ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 236ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 240ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 244ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned int*>(base + 248ull * cap)[idx] = R.r54;
            reinterpret_cast<unsigned int*>(base + 252ull * cap)[idx] = R.r55;
            reinterpret_cast<unsigned int*>(base + 256ull * cap)[idx] = R.r56;
            reinterpret_cast<unsigned*>(base + 260ull * cap)[idx] = tid;
            return;
        case 4: // shade
            reinterpret_cast<float*>(base + 264ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 268ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 272ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 276ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 280ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 284ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 288ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 292ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 296ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 300ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 304ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 308ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 312ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 316ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 320ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 324ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 328ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 332ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 336ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 340ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned int*>(base + 344ull * cap)[idx] = R.r54;
            reinterpret_cast<unsigned*>(base + 348ull * cap)[idx] = tid;
            return;
        case 5: // hitp
            reinterpret_cast<float*>(base + 352ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 356ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 360ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 364ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 368ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 372ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 376ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 380ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 384ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 388ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 392ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 396ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 400ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 404ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 408ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 412ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 416ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 420ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 424ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 428ull * cap)[idx] = R.r53;
            reinterpret_cast<unsigned int*>(base + 432ull * cap)[idx] = R.r54;
            reinterpret_cast<unsigned*>(base + 436ull * cap)[idx] = tid;
            return;
        case 6: // emit
            reinterpret_cast<float*>(base + 440ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 444ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 448ull * cap)[idx] = R.r5;
            reinterpret_cast<float*>(base + 452ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 456ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 460ull * cap)[idx] = R.r51;
            reinterpret_cast<float*>(base + 464ull * cap)[idx] = R.r76;
            reinterpret_cast<float*>(base + 468ull * cap)[idx] = R.r77;
            reinterpret_cast<float*>(base + 472ull * cap)[idx] = R.r78;
            reinterpret_cast<unsigned*>(base + 476ull * cap)[idx] = tid;
            return;
        case 7: // surf
            reinterpret_cast<float*>(base + 480ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 484ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 488ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 492ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 496ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 500ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 504ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 508ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 512ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 516ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 520ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 524ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 528ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 532ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 536ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 540ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 544ull * cap)[idx] = R.r76;
            reinterpret_cast<float*>(base + 548ull * cap)[idx] = R.r77;
            reinterpret_cast<float*>(base + 552ull * cap)[idx] = R.r78;
            reinterpret_cast<unsigned int*>(base + 556ull * cap)[idx] = R.r79;
            reinterpret_cast<float*>(base + 560ull * cap)[idx] = R.r80;
            reinterpret_cast<float*>(base + 564ull * cap)[idx] = R.r81;
            reinterpret_cast<float*>(base + 568ull * cap)[idx] = R.r82;
            reinterpret_cast<float*>(base + 572ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 576ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 580ull * cap)[idx] = R.r85;
            reinterpret_cast<unsigned*>(base + 584ull * cap)[idx] = tid;
            return;
        case 8: // rrchk
            reinterpret_cast<float*>(base + 592ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 596ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 600ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 604ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 608ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 612ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 616ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 620ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 624ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 628ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 632ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 636ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 640ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 644ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 648ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 652ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 656ull * cap)[idx] = R.r76;
            reinterpret_cast<float*>(base + 660ull * cap)[idx] = R.r77;
            reinterpret_cast<float*>(base + 664ull * cap)[idx] = R.r78;
            reinterpret_cast<unsigned int*>(base + 668ull * cap)[idx] = R.r79;
            reinterpret_cast<float*>(base + 672ull * cap)[idx] = R.r80;
            reinterpret_cast<float*>(base + 676ull * cap)[idx] = R.r81;
            reinterpret_cast<float*>(base + 680ull * cap)[idx] = R.r82;
            reinterpret_cast<float*>(base + 684ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 688ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 692ull * cap)[idx] = R.r85;
            reinterpret_cast<unsigned*>(base + 696ull * cap)[idx] = tid;
            return;
        case 9: // rr_roll
            reinterpret_cast<float*>(base + 704ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 708ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 712ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 716ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 720ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 724ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 728ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 732ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 736ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 740ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 744ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 748ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 752ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 756ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 760ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 764ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 768ull * cap)[idx] = R.r76;
            reinterpret_cast<float*>(base + 772ull * cap)[idx] = R.r77;
            reinterpret_cast<float*>(base + 776ull * cap)[idx] = R.r78;
            reinterpret_cast<unsigned int*>(base + 780ull * cap)[idx] = R.r79;
            reinterpret_cast<float*>(base + 784ull * cap)[idx] = R.r80;
            reinterpret_cast<float*>(base + 788ull * cap)[idx] = R.r81;
            reinterpret_cast<float*>(base + 792ull * cap)[idx] = R.r82;
            reinterpret_cast<float*>(base + 796ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 800ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 804ull * cap)[idx] = R.r85;
            reinterpret_cast<unsigned*>(base + 808ull * cap)[idx] = tid;
            return;
        case 10: // rr
            reinterpret_cast<float*>(base + 816ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 820ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 824ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 828ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 832ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 836ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 840ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 844ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 848ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 852ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 856ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 860ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 864ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 868ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 872ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 876ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 880ull * cap)[idx] = R.r76;
            reinterpret_cast<float*>(base + 884ull * cap)[idx] = R.r77;
            reinterpret_cast<float*>(base + 888ull * cap)[idx] = R.r78;
            reinterpret_cast<unsigned int*>(base + 892ull * cap)[idx] = R.r79;
            reinterpret_cast<float*>(base + 896ull * cap)[idx] = R.r80;
            reinterpret_cast<float*>(base + 900ull * cap)[idx] = R.r81;
            reinterpret_cast<float*>(base + 904ull * cap)[idx] = R.r82;
            reinterpret_cast<float*>(base + 908ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 912ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 916ull * cap)[idx] = R.r85;
            reinterpret_cast<unsigned int*>(base + 920ull * cap)[idx] = R.r130;
            reinterpret_cast<unsigned*>(base + 924ull * cap)[idx] = tid;
            return;
        case 11: // rr_keep
            reinterpret_cast<float*>(base + 928ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 932ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 936ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 940ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 944ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 948ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 952ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 956ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 960ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 964ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 968ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 972ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 976ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 980ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 984ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 988ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 992ull * cap)[idx] = R.r76;
            reinterpret_cast<float*>(base + 996ull * cap)[idx] = R.r77;
            reinterpret_cast<float*>(base + 1000ull * cap)[idx] = R.r78;
            reinterpret_cast<unsigned int*>(base + 1004ull * cap)[idx] = R.r79;
            reinterpret_cast<float*>(base + 1008ull * cap)[idx] = R.r80;
            reinterpret_cast<float*>(base + 1012ull * cap)[idx] = R.r81;
            reinterpret_cast<float*>(base + 1016ull * cap)[idx] = R.r82;
            reinterpret_cast<float*>(base + 1020ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 1024ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 1028ull * cap)[idx] = R.r85;
            reinterpret_cast<float*>(base + 1032ull * cap)[idx] = R.r86;
            reinterpret_cast<unsigned*>(base + 1036ull * cap)[idx] = tid;
            return;
        case 12: // scatter
            reinterpret_cast<float*>(base + 1040ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1044ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 1048ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1052ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 1056ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 1060ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1064ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 1068ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 1072ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 1076ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 1080ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 1084ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 1088ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 1092ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 1096ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 1100ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 1104ull * cap)[idx] = R.r76;
            reinterpret_cast<float*>(base + 1108ull * cap)[idx] = R.r77;
            reinterpret_cast<float*>(base + 1112ull * cap)[idx] = R.r78;
            reinterpret_cast<unsigned int*>(base + 1116ull * cap)[idx] = R.r79;
            reinterpret_cast<float*>(base + 1120ull * cap)[idx] = R.r80;
            reinterpret_cast<float*>(base + 1124ull * cap)[idx] = R.r81;
            reinterpret_cast<float*>(base + 1128ull * cap)[idx] = R.r82;
            reinterpret_cast<float*>(base + 1132ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 1136ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 1140ull * cap)[idx] = R.r85;
            reinterpret_cast<unsigned*>(base + 1144ull * cap)[idx] = tid;
            return;
        case 13: // mirror
            reinterpret_cast<float*>(base + 1152ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1156ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 1160ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1164ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 1168ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 1172ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1176ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 1180ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 1184ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 1188ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 1192ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 1196ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 1200ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 1204ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 1208ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 1212ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 1216ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 1220ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 1224ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 1228ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 1232ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 1236ull * cap)[idx] = R.r85;
            reinterpret_cast<float*>(base + 1240ull * cap)[idx] = R.r87;
            reinterpret_cast<unsigned*>(base + 1244ull * cap)[idx] = tid;
            return;
        case 14: // diffuse
            reinterpret_cast<float*>(base + 1248ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1252ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 1256ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1260ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 1264ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 1268ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1272ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 1276ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 1280ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 1284ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 1288ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 1292ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 1296ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 1300ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 1304ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 1308ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 1312ull * cap)[idx] = R.r92;
            reinterpret_cast<float*>(base + 1316ull * cap)[idx] = R.r93;
            reinterpret_cast<float*>(base + 1320ull * cap)[idx] = R.r94;
            reinterpret_cast<unsigned*>(base + 1324ull * cap)[idx] = tid;
            return;
        case 15: // disk_roll
            reinterpret_cast<float*>(base + 1328ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1332ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 1336ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1340ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 1344ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 1348ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1352ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 1356ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 1360ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 1364ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 1368ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 1372ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 1376ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 1380ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 1384ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 1388ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 1392ull * cap)[idx] = R.r92;
            reinterpret_cast<float*>(base + 1396ull * cap)[idx] = R.r93;
            reinterpret_cast<float*>(base + 1400ull * cap)[idx] = R.r94;
            reinterpret_cast<float*>(base + 1404ull * cap)[idx] = R.r100;
            reinterpret_cast<float*>(base + 1408ull * cap)[idx] = R.r101;
            reinterpret_cast<float*>(base + 1412ull * cap)[idx] = R.r102;
            reinterpret_cast<float*>(base + 1416ull * cap)[idx] = R.r103;
            reinterpret_cast<float*>(base + 1420ull * cap)[idx] = R.r104;
            reinterpret_cast<float*>(base + 1424ull * cap)[idx] = R.r105;
            reinterpret_cast<unsigned*>(base + 1428ull * cap)[idx] = tid;
            return;
        case 16: // disk
            reinterpret_cast<float*>(base + 1432ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1436ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 1440ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1444ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 1448ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 1452ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1456ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 1460ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 1464ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 1468ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 1472ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 1476ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 1480ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 1484ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 1488ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 1492ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 1496ull * cap)[idx] = R.r92;
            reinterpret_cast<float*>(base + 1500ull * cap)[idx] = R.r93;
            reinterpret_cast<float*>(base + 1504ull * cap)[idx] = R.r94;
            reinterpret_cast<float*>(base + 1508ull * cap)[idx] = R.r100;
            reinterpret_cast<float*>(base + 1512ull * cap)[idx] = R.r101;
            reinterpret_cast<float*>(base + 1516ull * cap)[idx] = R.r102;
            reinterpret_cast<float*>(base + 1520ull * cap)[idx] = R.r103;
            reinterpret_cast<float*>(base + 1524ull * cap)[idx] = R.r104;
            reinterpret_cast<float*>(base + 1528ull * cap)[idx] = R.r105;
            reinterpret_cast<unsigned int*>(base + 1532ull * cap)[idx] = R.r130;
            reinterpret_cast<unsigned int*>(base + 1536ull * cap)[idx] = R.r131;
            reinterpret_cast<unsigned*>(base + 1540ull * cap)[idx] = tid;
            return;
        case 17: // disk_ok
            reinterpret_cast<float*>(base + 1544ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1548ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 1552ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1556ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 1560ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 1564ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1568ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 1572ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 1576ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 1580ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 1584ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 1588ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 1592ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 1596ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 1600ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 1604ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 1608ull * cap)[idx] = R.r92;
            reinterpret_cast<float*>(base + 1612ull * cap)[idx] = R.r93;
            reinterpret_cast<float*>(base + 1616ull * cap)[idx] = R.r94;
            reinterpret_cast<float*>(base + 1620ull * cap)[idx] = R.r100;
            reinterpret_cast<float*>(base + 1624ull * cap)[idx] = R.r101;
            reinterpret_cast<float*>(base + 1628ull * cap)[idx] = R.r102;
            reinterpret_cast<float*>(base + 1632ull * cap)[idx] = R.r103;
            reinterpret_cast<float*>(base + 1636ull * cap)[idx] = R.r104;
            reinterpret_cast<float*>(base + 1640ull * cap)[idx] = R.r105;
            reinterpret_cast<float*>(base + 1644ull * cap)[idx] = R.r106;
            reinterpret_cast<float*>(base + 1648ull * cap)[idx] = R.r107;
            reinterpret_cast<float*>(base + 1652ull * cap)[idx] = R.r108;
            reinterpret_cast<unsigned*>(base + 1656ull * cap)[idx] = tid;
            return;
        case 18: // glass
            reinterpret_cast<float*>(base + 1664ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1668ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 1672ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1676ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 1680ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 1684ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1688ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 1692ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 1696ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 1700ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 1704ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 1708ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 1712ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 1716ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 1720ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 1724ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 1728ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 1732ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 1736ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 1740ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 1744ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 1748ull * cap)[idx] = R.r85;
            reinterpret_cast<float*>(base + 1752ull * cap)[idx] = R.r87;
            reinterpret_cast<unsigned int*>(base + 1756ull * cap)[idx] = R.r88;
            reinterpret_cast<float*>(base + 1760ull * cap)[idx] = R.r92;
            reinterpret_cast<float*>(base + 1764ull * cap)[idx] = R.r93;
            reinterpret_cast<float*>(base + 1768ull * cap)[idx] = R.r94;
            reinterpret_cast<unsigned*>(base + 1772ull * cap)[idx] = tid;
            return;
        case 19: // refr
            reinterpret_cast<float*>(base + 1776ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1780ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 1784ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1788ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 1792ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 1796ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1800ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 1804ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 1808ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 1812ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 1816ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 1820ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 1824ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 1828ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 1832ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 1836ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 1840ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 1844ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 1848ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 1852ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 1856ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 1860ull * cap)[idx] = R.r85;
            reinterpret_cast<float*>(base + 1864ull * cap)[idx] = R.r87;
            reinterpret_cast<unsigned int*>(base + 1868ull * cap)[idx] = R.r88;
            reinterpret_cast<float*>(base + 1872ull * cap)[idx] = R.r111;
            reinterpret_cast<float*>(base + 1876ull * cap)[idx] = R.r112;
            reinterpret_cast<float*>(base + 1880ull * cap)[idx] = R.r113;
            reinterpret_cast<unsigned*>(base + 1884ull * cap)[idx] = tid;
            return;
        case 20: // fres
            reinterpret_cast<float*>(base + 1888ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 1892ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 1896ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 1900ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 1904ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 1908ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 1912ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 1916ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 1920ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 1924ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 1928ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 1932ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 1936ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 1940ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 1944ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 1948ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 1952ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 1956ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 1960ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 1964ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 1968ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 1972ull * cap)[idx] = R.r85;
            reinterpret_cast<float*>(base + 1976ull * cap)[idx] = R.r87;
            reinterpret_cast<float*>(base + 1980ull * cap)[idx] = R.r117;
            reinterpret_cast<float*>(base + 1984ull * cap)[idx] = R.r118;
            reinterpret_cast<float*>(base + 1988ull * cap)[idx] = R.r119;
            reinterpret_cast<float*>(base + 1992ull * cap)[idx] = R.r127;
            reinterpret_cast<float*>(base + 1996ull * cap)[idx] = R.r128;
            reinterpret_cast<float*>(base + 2000ull * cap)[idx] = R.r129;
            reinterpret_cast<unsigned int*>(base + 2004ull * cap)[idx] = R.r130;
            reinterpret_cast<unsigned*>(base + 2008ull * cap)[idx] = tid;
            return;
        case 21: // take_refl
            reinterpret_cast<float*>(base + 2016ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2020ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 2024ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2028ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 2032ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 2036ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 2040ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 2044ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 2048ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 2052ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 2056ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 2060ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 2064ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 2068ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 2072ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 2076ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 2080ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 2084ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 2088ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 2092ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 2096ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 2100ull * cap)[idx] = R.r85;
            reinterpret_cast<float*>(base + 2104ull * cap)[idx] = R.r87;
            reinterpret_cast<float*>(base + 2108ull * cap)[idx] = R.r128;
            reinterpret_cast<unsigned*>(base + 2112ull * cap)[idx] = tid;
            return;
        case 22: // take_refr
            reinterpret_cast<float*>(base + 2120ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2124ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 2128ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2132ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 2136ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 2140ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 2144ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 2148ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 2152ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 2156ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 2160ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 2164ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 2168ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 2172ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 2176ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 2180ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 2184ull * cap)[idx] = R.r117;
            reinterpret_cast<float*>(base + 2188ull * cap)[idx] = R.r118;
            reinterpret_cast<float*>(base + 2192ull * cap)[idx] = R.r119;
            reinterpret_cast<float*>(base + 2196ull * cap)[idx] = R.r129;
            reinterpret_cast<unsigned*>(base + 2200ull * cap)[idx] = tid;
            return;
        case 23: // roll
            reinterpret_cast<float*>(base + 2208ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2212ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 2216ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2220ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2224ull * cap)[idx] = R.r9;
            reinterpret_cast<unsigned int*>(base + 2228ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 2232ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 2236ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 2240ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 2244ull * cap)[idx] = R.r15;
            reinterpret_cast<float*>(base + 2248ull * cap)[idx] = R.r16;
            reinterpret_cast<float*>(base + 2252ull * cap)[idx] = R.r17;
            reinterpret_cast<unsigned int*>(base + 2256ull * cap)[idx] = R.r20;
            reinterpret_cast<unsigned int*>(base + 2260ull * cap)[idx] = R.r21;
            reinterpret_cast<unsigned int*>(base + 2264ull * cap)[idx] = R.r22;
            reinterpret_cast<unsigned int*>(base + 2268ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 2272ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 2276ull * cap)[idx] = R.r25;
            reinterpret_cast<unsigned int*>(base + 2280ull * cap)[idx] = R.r26;
            reinterpret_cast<float*>(base + 2284ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 2288ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 2292ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 2296ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 2300ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 2304ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 2308ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 2312ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 2316ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 2320ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 2324ull * cap)[idx] = R.r76;
            reinterpret_cast<float*>(base + 2328ull * cap)[idx] = R.r77;
            reinterpret_cast<float*>(base + 2332ull * cap)[idx] = R.r78;
            reinterpret_cast<unsigned int*>(base + 2336ull * cap)[idx] = R.r79;
            reinterpret_cast<float*>(base + 2340ull * cap)[idx] = R.r80;
            reinterpret_cast<float*>(base + 2344ull * cap)[idx] = R.r81;
            reinterpret_cast<float*>(base + 2348ull * cap)[idx] = R.r82;
            reinterpret_cast<float*>(base + 2352ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 2356ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 2360ull * cap)[idx] = R.r85;
            reinterpret_cast<float*>(base + 2364ull * cap)[idx] = R.r87;
            reinterpret_cast<float*>(base + 2368ull * cap)[idx] = R.r92;
            reinterpret_cast<float*>(base + 2372ull * cap)[idx] = R.r93;
            reinterpret_cast<float*>(base + 2376ull * cap)[idx] = R.r94;
            reinterpret_cast<float*>(base + 2380ull * cap)[idx] = R.r100;
            reinterpret_cast<float*>(base + 2384ull * cap)[idx] = R.r101;
            reinterpret_cast<float*>(base + 2388ull * cap)[idx] = R.r102;
            reinterpret_cast<float*>(base + 2392ull * cap)[idx] = R.r103;
            reinterpret_cast<float*>(base + 2396ull * cap)[idx] = R.r104;
            reinterpret_cast<float*>(base + 2400ull * cap)[idx] = R.r105;
            reinterpret_cast<float*>(base + 2404ull * cap)[idx] = R.r117;
            reinterpret_cast<float*>(base + 2408ull * cap)[idx] = R.r118;
            reinterpret_cast<float*>(base + 2412ull * cap)[idx] = R.r119;
            reinterpret_cast<float*>(base + 2416ull * cap)[idx] = R.r127;
            reinterpret_cast<float*>(base + 2420ull * cap)[idx] = R.r128;
            reinterpret_cast<float*>(base + 2424ull * cap)[idx] = R.r129;
            reinterpret_cast<unsigned*>(base + 2428ull * cap)[idx] = tid;
            return;
        case 24: // roll, context 0
            reinterpret_cast<unsigned int*>(base + 2432ull * cap)[idx] = R.r7;
            reinterpret_cast<unsigned int*>(base + 2436ull * cap)[idx] = R.r9;
            reinterpret_cast<unsigned int*>(base + 2440ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 2444ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 2448ull * cap)[idx] = R.r13;
            reinterpret_cast<float*>(base + 2452ull * cap)[idx] = R.r14;
            reinterpret_cast<float*>(base + 2456ull * cap)[idx] = R.r15;
            reinterpret_cast<float*>(base + 2460ull * cap)[idx] = R.r16;
            reinterpret_cast<float*>(base + 2464ull * cap)[idx] = R.r17;
            reinterpret_cast<unsigned int*>(base + 2468ull * cap)[idx] = R.r20;
            reinterpret_cast<unsigned int*>(base + 2472ull * cap)[idx] = R.r21;
            reinterpret_cast<unsigned int*>(base + 2476ull * cap)[idx] = R.r22;
            reinterpret_cast<unsigned int*>(base + 2480ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 2484ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 2488ull * cap)[idx] = R.r25;
            reinterpret_cast<unsigned*>(base + 2492ull * cap)[idx] = tid;
            return;
        case 25: // roll, context 1
            reinterpret_cast<float*>(base + 2496ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2500ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 2504ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2508ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 2512ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 2516ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 2520ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 2524ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 2528ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 2532ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 2536ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 2540ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 2544ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 2548ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 2552ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 2556ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 2560ull * cap)[idx] = R.r76;
            reinterpret_cast<float*>(base + 2564ull * cap)[idx] = R.r77;
            reinterpret_cast<float*>(base + 2568ull * cap)[idx] = R.r78;
            reinterpret_cast<unsigned int*>(base + 2572ull * cap)[idx] = R.r79;
            reinterpret_cast<float*>(base + 2576ull * cap)[idx] = R.r80;
            reinterpret_cast<float*>(base + 2580ull * cap)[idx] = R.r81;
            reinterpret_cast<float*>(base + 2584ull * cap)[idx] = R.r82;
            reinterpret_cast<float*>(base + 2588ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 2592ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 2596ull * cap)[idx] = R.r85;
            reinterpret_cast<unsigned*>(base + 2600ull * cap)[idx] = tid;
            return;
        case 26: // roll, context 2
            reinterpret_cast<float*>(base + 2608ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2612ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 2616ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2620ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 2624ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 2628ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 2632ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 2636ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 2640ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 2644ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 2648ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 2652ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 2656ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 2660ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 2664ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 2668ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 2672ull * cap)[idx] = R.r92;
            reinterpret_cast<float*>(base + 2676ull * cap)[idx] = R.r93;
            reinterpret_cast<float*>(base + 2680ull * cap)[idx] = R.r94;
            reinterpret_cast<float*>(base + 2684ull * cap)[idx] = R.r100;
            reinterpret_cast<float*>(base + 2688ull * cap)[idx] = R.r101;
            reinterpret_cast<float*>(base + 2692ull * cap)[idx] = R.r102;
            reinterpret_cast<float*>(base + 2696ull * cap)[idx] = R.r103;
            reinterpret_cast<float*>(base + 2700ull * cap)[idx] = R.r104;
            reinterpret_cast<float*>(base + 2704ull * cap)[idx] = R.r105;
            reinterpret_cast<unsigned*>(base + 2708ull * cap)[idx] = tid;
            return;
        case 27: // roll, context 3
            reinterpret_cast<float*>(base + 2712ull * cap)[idx] = R.r3;
            reinterpret_cast<float*>(base + 2716ull * cap)[idx] = R.r4;
            reinterpret_cast<float*>(base + 2720ull * cap)[idx] = R.r5;
            reinterpret_cast<unsigned int*>(base + 2724ull * cap)[idx] = R.r11;
            reinterpret_cast<unsigned int*>(base + 2728ull * cap)[idx] = R.r12;
            reinterpret_cast<unsigned int*>(base + 2732ull * cap)[idx] = R.r13;
            reinterpret_cast<unsigned int*>(base + 2736ull * cap)[idx] = R.r23;
            reinterpret_cast<unsigned int*>(base + 2740ull * cap)[idx] = R.r24;
            reinterpret_cast<unsigned int*>(base + 2744ull * cap)[idx] = R.r25;
            reinterpret_cast<float*>(base + 2748ull * cap)[idx] = R.r42;
            reinterpret_cast<float*>(base + 2752ull * cap)[idx] = R.r43;
            reinterpret_cast<float*>(base + 2756ull * cap)[idx] = R.r44;
            reinterpret_cast<float*>(base + 2760ull * cap)[idx] = R.r46;
            reinterpret_cast<float*>(base + 2764ull * cap)[idx] = R.r47;
            reinterpret_cast<float*>(base + 2768ull * cap)[idx] = R.r48;
            reinterpret_cast<float*>(base + 2772ull * cap)[idx] = R.r49;
            reinterpret_cast<float*>(base + 2776ull * cap)[idx] = R.r50;
            reinterpret_cast<float*>(base + 2780ull * cap)[idx] = R.r51;
            reinterpret_cast<unsigned int*>(base + 2784ull * cap)[idx] = R.r52;
            reinterpret_cast<float*>(base + 2788ull * cap)[idx] = R.r83;
            reinterpret_cast<float*>(base + 2792ull * cap)[idx] = R.r84;
            reinterpret_cast<float*>(base + 2796ull * cap)[idx] = R.r85;
            reinterpret_cast<float*>(base + 2800ull * cap)[idx] = R.r87;
            reinterpret_cast<float*>(base + 2804ull * cap)[idx] = R.r117;
            reinterpret_cast<float*>(base + 2808ull * cap)[idx] = R.r118;
            reinterpret_cast<float*>(base + 2812ull * cap)[idx] = R.r119;
            reinterpret_cast<float*>(base + 2816ull * cap)[idx] = R.r127;
            reinterpret_cast<float*>(base + 2820ull * cap)[idx] = R.r128;
            reinterpret_cast<float*>(base + 2824ull * cap)[idx] = R.r129;
            reinterpret_cast<unsigned*>(base + 2828ull * cap)[idx] = tid;
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
            R.r2 = reinterpret_cast<const unsigned int*>(base + 4ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 8ull * cap)[idx];
        case 1: // prim
            R.r7 = reinterpret_cast<const unsigned int*>(base + 16ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 20ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 24ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 28ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 32ull * cap)[idx];
            R.r14 = reinterpret_cast<const float*>(base + 36ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 40ull * cap)[idx];
            R.r16 = reinterpret_cast<const float*>(base + 44ull * cap)[idx];
            R.r17 = reinterpret_cast<const float*>(base + 48ull * cap)[idx];
            R.r20 = reinterpret_cast<const unsigned int*>(base + 52ull * cap)[idx];
            R.r21 = reinterpret_cast<const unsigned int*>(base + 56ull * cap)[idx];
            R.r22 = reinterpret_cast<const unsigned int*>(base + 60ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 64ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 68ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 72ull * cap)[idx];
            R.r130 = reinterpret_cast<const unsigned int*>(base + 76ull * cap)[idx];
            R.r131 = reinterpret_cast<const unsigned int*>(base + 80ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 84ull * cap)[idx];
        case 2: // bounce
            R.r3 = reinterpret_cast<const float*>(base + 88ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 92ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 96ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 100ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 104ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 108ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 112ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 116ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 120ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 124ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 128ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 132ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 136ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 140ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 144ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 148ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 152ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 156ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 160ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 164ull * cap)[idx];
        case 3: // isect
            R.r3 = reinterpret_cast<const float*>(base + 168ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 172ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 176ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 180ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 184ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 188ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 192ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 196ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 200ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 204ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 208ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 212ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 216ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 220ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 224ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 228ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 232ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 236ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 240ull * cap)[idx];
            R.r53 = reinterpret_cast<const float*>(base + 244ull * cap)[idx];
            R.r54 = reinterpret_cast<const unsigned int*>(base + 248ull * cap)[idx];
            R.r55 = reinterpret_cast<const unsigned int*>(base + 252ull * cap)[idx];
            R.r56 = reinterpret_cast<const unsigned int*>(base + 256ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 260ull * cap)[idx];
        case 4: // shade
            R.r3 = reinterpret_cast<const float*>(base + 264ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 268ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 272ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 276ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 280ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 284ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 288ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 292ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 296ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 300ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 304ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 308ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 312ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 316ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 320ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 324ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 328ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 332ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 336ull * cap)[idx];
            R.r53 = reinterpret_cast<const float*>(base + 340ull * cap)[idx];
            R.r54 = reinterpret_cast<const unsigned int*>(base + 344ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 348ull * cap)[idx];
        case 5: // hitp
            R.r3 = reinterpret_cast<const float*>(base + 352ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 356ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 360ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 364ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 368ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 372ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 376ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 380ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 384ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 388ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 392ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 396ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 400ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 404ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 408ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 412ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 416ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 420ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 424ull * cap)[idx];
            R.r53 = reinterpret_cast<const float*>(base + 428ull * cap)[idx];
            R.r54 = reinterpret_cast<const unsigned int*>(base + 432ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 436ull * cap)[idx];
        case 6: // emit
            R.r3 = reinterpret_cast<const float*>(base + 440ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 444ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 448ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 452ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 456ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 460ull * cap)[idx];
            R.r76 = reinterpret_cast<const float*>(base + 464ull * cap)[idx];
            R.r77 = reinterpret_cast<const float*>(base + 468ull * cap)[idx];
            R.r78 = reinterpret_cast<const float*>(base + 472ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 476ull * cap)[idx];
        case 7: // surf
            R.r3 = reinterpret_cast<const float*>(base + 480ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 484ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 488ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 492ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 496ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 500ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 504ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 508ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 512ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 516ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 520ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 524ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 528ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 532ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 536ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 540ull * cap)[idx];
            R.r76 = reinterpret_cast<const float*>(base + 544ull * cap)[idx];
            R.r77 = reinterpret_cast<const float*>(base + 548ull * cap)[idx];
            R.r78 = reinterpret_cast<const float*>(base + 552ull * cap)[idx];
            R.r79 = reinterpret_cast<const unsigned int*>(base + 556ull * cap)[idx];
            R.r80 = reinterpret_cast<const float*>(base + 560ull * cap)[idx];
            R.r81 = reinterpret_cast<const float*>(base + 564ull * cap)[idx];
            R.r82 = reinterpret_cast<const float*>(base + 568ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 572ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 576ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 580ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 584ull * cap)[idx];
        case 8: // rrchk
            R.r3 = reinterpret_cast<const float*>(base + 592ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 596ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 600ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 604ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 608ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 612ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 616ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 620ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 624ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 628ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 632ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 636ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 640ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 644ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 648ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 652ull * cap)[idx];
            R.r76 = reinterpret_cast<const float*>(base + 656ull * cap)[idx];
            R.r77 = reinterpret_cast<const float*>(base + 660ull * cap)[idx];
            R.r78 = reinterpret_cast<const float*>(base + 664ull * cap)[idx];
            R.r79 = reinterpret_cast<const unsigned int*>(base + 668ull * cap)[idx];
            R.r80 = reinterpret_cast<const float*>(base + 672ull * cap)[idx];
            R.r81 = reinterpret_cast<const float*>(base + 676ull * cap)[idx];
            R.r82 = reinterpret_cast<const float*>(base + 680ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 684ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 688ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 692ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 696ull * cap)[idx];
        case 9: // rr_roll
            R.r3 = reinterpret_cast<const float*>(base + 704ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 708ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 712ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 716ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 720ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 724ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 728ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 732ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 736ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 740ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 744ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 748ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 752ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 756ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 760ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 764ull * cap)[idx];
            R.r76 = reinterpret_cast<const float*>(base + 768ull * cap)[idx];
            R.r77 = reinterpret_cast<const float*>(base + 772ull * cap)[idx];
            R.r78 = reinterpret_cast<const float*>(base + 776ull * cap)[idx];
            R.r79 = reinterpret_cast<const unsigned int*>(base + 780ull * cap)[idx];
            R.r80 = reinterpret_cast<const float*>(base + 784ull * cap)[idx];
            R.r81 = reinterpret_cast<const float*>(base + 788ull * cap)[idx];
            R.r82 = reinterpret_cast<const float*>(base + 792ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 796ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 800ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 804ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 808ull * cap)[idx];
        case 10: // rr
            R.r3 = reinterpret_cast<const float*>(base + 816ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 820ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 824ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 828ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 832ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 836ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 840ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 844ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 848ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 852ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 856ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 860ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 864ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 868ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 872ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 876ull * cap)[idx];
            R.r76 = reinterpret_cast<const float*>(base + 880ull * cap)[idx];
            R.r77 = reinterpret_cast<const float*>(base + 884ull * cap)[idx];
            R.r78 = reinterpret_cast<const float*>(base + 888ull * cap)[idx];
            R.r79 = reinterpret_cast<const unsigned int*>(base + 892ull * cap)[idx];
            R.r80 = reinterpret_cast<const float*>(base + 896ull * cap)[idx];
            R.r81 = reinterpret_cast<const float*>(base + 900ull * cap)[idx];
            R.r82 = reinterpret_cast<const float*>(base + 904ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 908ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 912ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 916ull * cap)[idx];
            R.r130 = reinterpret_cast<const unsigned int*>(base + 920ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 924ull * cap)[idx];
        case 11: // rr_keep
            R.r3 = reinterpret_cast<const float*>(base + 928ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 932ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 936ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 940ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 944ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 948ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 952ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 956ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 960ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 964ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 968ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 972ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 976ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 980ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 984ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 988ull * cap)[idx];
            R.r76 = reinterpret_cast<const float*>(base + 992ull * cap)[idx];
            R.r77 = reinterpret_cast<const float*>(base + 996ull * cap)[idx];
            R.r78 = reinterpret_cast<const float*>(base + 1000ull * cap)[idx];
            R.r79 = reinterpret_cast<const unsigned int*>(base + 1004ull * cap)[idx];
            R.r80 = reinterpret_cast<const float*>(base + 1008ull * cap)[idx];
            R.r81 = reinterpret_cast<const float*>(base + 1012ull * cap)[idx];
            R.r82 = reinterpret_cast<const float*>(base + 1016ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 1020ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 1024ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 1028ull * cap)[idx];
            R.r86 = reinterpret_cast<const float*>(base + 1032ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1036ull * cap)[idx];
        case 12: // scatter
            R.r3 = reinterpret_cast<const float*>(base + 1040ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1044ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 1048ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 1052ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 1056ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 1060ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 1064ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 1068ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 1072ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 1076ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 1080ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 1084ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 1088ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 1092ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 1096ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 1100ull * cap)[idx];
            R.r76 = reinterpret_cast<const float*>(base + 1104ull * cap)[idx];
            R.r77 = reinterpret_cast<const float*>(base + 1108ull * cap)[idx];
            R.r78 = reinterpret_cast<const float*>(base + 1112ull * cap)[idx];
            R.r79 = reinterpret_cast<const unsigned int*>(base + 1116ull * cap)[idx];
            R.r80 = reinterpret_cast<const float*>(base + 1120ull * cap)[idx];
            R.r81 = reinterpret_cast<const float*>(base + 1124ull * cap)[idx];
            R.r82 = reinterpret_cast<const float*>(base + 1128ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 1132ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 1136ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 1140ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1144ull * cap)[idx];
        case 13: // mirror
            R.r3 = reinterpret_cast<const float*>(base + 1152ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1156ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 1160ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 1164ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 1168ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 1172ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 1176ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 1180ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 1184ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 1188ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 1192ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 1196ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 1200ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 1204ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 1208ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 1212ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 1216ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 1220ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 1224ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 1228ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 1232ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 1236ull * cap)[idx];
            R.r87 = reinterpret_cast<const float*>(base + 1240ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1244ull * cap)[idx];
        case 14: // diffuse
            R.r3 = reinterpret_cast<const float*>(base + 1248ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1252ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 1256ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 1260ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 1264ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 1268ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 1272ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 1276ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 1280ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 1284ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 1288ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 1292ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 1296ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 1300ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 1304ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 1308ull * cap)[idx];
            R.r92 = reinterpret_cast<const float*>(base + 1312ull * cap)[idx];
            R.r93 = reinterpret_cast<const float*>(base + 1316ull * cap)[idx];
            R.r94 = reinterpret_cast<const float*>(base + 1320ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1324ull * cap)[idx];
        case 15: // disk_roll
            R.r3 = reinterpret_cast<const float*>(base + 1328ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1332ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 1336ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 1340ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 1344ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 1348ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 1352ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 1356ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 1360ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 1364ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 1368ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 1372ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 1376ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 1380ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 1384ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 1388ull * cap)[idx];
            R.r92 = reinterpret_cast<const float*>(base + 1392ull * cap)[idx];
            R.r93 = reinterpret_cast<const float*>(base + 1396ull * cap)[idx];
            R.r94 = reinterpret_cast<const float*>(base + 1400ull * cap)[idx];
            R.r100 = reinterpret_cast<const float*>(base + 1404ull * cap)[idx];
            R.r101 = reinterpret_cast<const float*>(base + 1408ull * cap)[idx];
            R.r102 = reinterpret_cast<const float*>(base + 1412ull * cap)[idx];
            R.r103 = reinterpret_cast<const float*>(base + 1416ull * cap)[idx];
            R.r104 = reinterpret_cast<const float*>(base + 1420ull * cap)[idx];
            R.r105 = reinterpret_cast<const float*>(base + 1424ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1428ull * cap)[idx];
        case 16: // disk
            R.r3 = reinterpret_cast<const float*>(base + 1432ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1436ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 1440ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 1444ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 1448ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 1452ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 1456ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 1460ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 1464ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 1468ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 1472ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 1476ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 1480ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 1484ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 1488ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 1492ull * cap)[idx];
            R.r92 = reinterpret_cast<const float*>(base + 1496ull * cap)[idx];
            R.r93 = reinterpret_cast<const float*>(base + 1500ull * cap)[idx];
            R.r94 = reinterpret_cast<const float*>(base + 1504ull * cap)[idx];
            R.r100 = reinterpret_cast<const float*>(base + 1508ull * cap)[idx];
            R.r101 = reinterpret_cast<const float*>(base + 1512ull * cap)[idx];
            R.r102 = reinterpret_cast<const float*>(base + 1516ull * cap)[idx];
            R.r103 = reinterpret_cast<const float*>(base + 1520ull * cap)[idx];
            R.r104 = reinterpret_cast<const float*>(base + 1524ull * cap)[idx];
            R.r105 = reinterpret_cast<const float*>(base + 1528ull * cap)[idx];
            R.r130 = reinterpret_cast<const unsigned int*>(base + 1532ull * cap)[idx];
            R.r131 = reinterpret_cast<const unsigned int*>(base + 1536ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1540ull * cap)[idx];
        case 17: // disk_ok
            R.r3 = reinterpret_cast<const float*>(base + 1544ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1548ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 1552ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 1556ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 1560ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 1564ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 1568ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 1572ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 1576ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 1580ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 1584ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 1588ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 1592ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 1596ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 1600ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 1604ull * cap)[idx];
            R.r92 = reinterpret_cast<const float*>(base + 1608ull * cap)[idx];
            R.r93 = reinterpret_cast<const float*>(base + 1612ull * cap)[idx];
            R.r94 = reinterpret_cast<const float*>(base + 1616ull * cap)[idx];
            R.r100 = reinterpret_cast<const float*>(base + 1620ull * cap)[idx];
            R.r101 = reinterpret_cast<const float*>(base + 1624ull * cap)[idx];
            R.r102 = reinterpret_cast<const float*>(base + 1628ull * cap)[idx];
            R.r103 = reinterpret_cast<const float*>(base + 1632ull * cap)[idx];
            R.r104 = reinterpret_cast<const float*>(base + 1636ull * cap)[idx];
            R.r105 = reinterpret_cast<const float*>(base + 1640ull * cap)[idx];
            R.r106 = reinterpret_cast<const float*>(base + 1644ull * cap)[idx];
            R.r107 = reinterpret_cast<const float*>(base + 1648ull * cap)[idx];
            R.r108 = reinterpret_cast<const float*>(base + 1652ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1656ull * cap)[idx];
        case 18: // glass
            R.r3 = reinterpret_cast<const float*>(base + 1664ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1668ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 1672ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 1676ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 1680ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 1684ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 1688ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 1692ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 1696ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 1700ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 1704ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 1708ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 1712ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 1716ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 1720ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 1724ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 1728ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 1732ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 1736ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 1740ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 1744ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 1748ull * cap)[idx];
            R.r87 = reinterpret_cast<const float*>(base + 1752ull * cap)[idx];
            R.r88 = reinterpret_cast<const unsigned int*>(base + 1756ull * cap)[idx];
            R.r92 = reinterpret_cast<const float*>(base + 1760ull * cap)[idx];
            R.r93 = reinterpret_cast<const float*>(base + 1764ull * cap)[idx];
            R.r94 = reinterpret_cast<const float*>(base + 1768ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1772ull * cap)[idx];
        case 19: // refr
            R.r3 = reinterpret_cast<const float*>(base + 1776ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1780ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 1784ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 1788ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 1792ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 1796ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 1800ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 1804ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 1808ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 1812ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 1816ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 1820ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 1824ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 1828ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 1832ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 1836ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 1840ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 1844ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 1848ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 1852ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 1856ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 1860ull * cap)[idx];
            R.r87 = reinterpret_cast<const float*>(base + 1864ull * cap)[idx];
            R.r88 = reinterpret_cast<const unsigned int*>(base + 1868ull * cap)[idx];
            R.r111 = reinterpret_cast<const float*>(base + 1872ull * cap)[idx];
            R.r112 = reinterpret_cast<const float*>(base + 1876ull * cap)[idx];
            R.r113 = reinterpret_cast<const float*>(base + 1880ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 1884ull * cap)[idx];
        case 20: // fres
            R.r3 = reinterpret_cast<const float*>(base + 1888ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 1892ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 1896ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 1900ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 1904ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 1908ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 1912ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 1916ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 1920ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 1924ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 1928ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 1932ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 1936ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 1940ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 1944ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 1948ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 1952ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 1956ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 1960ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 1964ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 1968ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 1972ull * cap)[idx];
            R.r87 = reinterpret_cast<const float*>(base + 1976ull * cap)[idx];
            R.r117 = reinterpret_cast<const float*>(base + 1980ull * cap)[idx];
            R.r118 = reinterpret_cast<const float*>(base + 1984ull * cap)[idx];
            R.r119 = reinterpret_cast<const float*>(base + 1988ull * cap)[idx];
            R.r127 = reinterpret_cast<const float*>(base + 1992ull * cap)[idx];
            R.r128 = reinterpret_cast<const float*>(base + 1996ull * cap)[idx];
            R.r129 = reinterpret_cast<const float*>(base + 2000ull * cap)[idx];
            R.r130 = reinterpret_cast<const unsigned int*>(base + 2004ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2008ull * cap)[idx];
        case 21: // take_refl
            R.r3 = reinterpret_cast<const float*>(base + 2016ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2020ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 2024ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 2028ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 2032ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 2036ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 2040ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 2044ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 2048ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 2052ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 2056ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 2060ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 2064ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 2068ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 2072ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 2076ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 2080ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 2084ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 2088ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 2092ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 2096ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 2100ull * cap)[idx];
            R.r87 = reinterpret_cast<const float*>(base + 2104ull * cap)[idx];
            R.r128 = reinterpret_cast<const float*>(base + 2108ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2112ull * cap)[idx];
        case 22: // take_refr
            R.r3 = reinterpret_cast<const float*>(base + 2120ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2124ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 2128ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 2132ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 2136ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 2140ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 2144ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 2148ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 2152ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 2156ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 2160ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 2164ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 2168ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 2172ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 2176ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 2180ull * cap)[idx];
            R.r117 = reinterpret_cast<const float*>(base + 2184ull * cap)[idx];
            R.r118 = reinterpret_cast<const float*>(base + 2188ull * cap)[idx];
            R.r119 = reinterpret_cast<const float*>(base + 2192ull * cap)[idx];
            R.r129 = reinterpret_cast<const float*>(base + 2196ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2200ull * cap)[idx];
        case 23: // roll
            R.r3 = reinterpret_cast<const float*>(base + 2208ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2212ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 2216ull * cap)[idx];
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2220ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2224ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 2228ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 2232ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 2236ull * cap)[idx];
            R.r14 = reinterpret_cast<const float*>(base + 2240ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2244ull * cap)[idx];
            R.r16 = reinterpret_cast<const float*>(base + 2248ull * cap)[idx];
            R.r17 = reinterpret_cast<const float*>(base + 2252ull * cap)[idx];
            R.r20 = reinterpret_cast<const unsigned int*>(base + 2256ull * cap)[idx];
            R.r21 = reinterpret_cast<const unsigned int*>(base + 2260ull * cap)[idx];
            R.r22 = reinterpret_cast<const unsigned int*>(base + 2264ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 2268ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 2272ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 2276ull * cap)[idx];
            R.r26 = reinterpret_cast<const unsigned int*>(base + 2280ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 2284ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 2288ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 2292ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 2296ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 2300ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 2304ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 2308ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 2312ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 2316ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 2320ull * cap)[idx];
            R.r76 = reinterpret_cast<const float*>(base + 2324ull * cap)[idx];
            R.r77 = reinterpret_cast<const float*>(base + 2328ull * cap)[idx];
            R.r78 = reinterpret_cast<const float*>(base + 2332ull * cap)[idx];
            R.r79 = reinterpret_cast<const unsigned int*>(base + 2336ull * cap)[idx];
            R.r80 = reinterpret_cast<const float*>(base + 2340ull * cap)[idx];
            R.r81 = reinterpret_cast<const float*>(base + 2344ull * cap)[idx];
            R.r82 = reinterpret_cast<const float*>(base + 2348ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 2352ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 2356ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 2360ull * cap)[idx];
            R.r87 = reinterpret_cast<const float*>(base + 2364ull * cap)[idx];
            R.r92 = reinterpret_cast<const float*>(base + 2368ull * cap)[idx];
            R.r93 = reinterpret_cast<const float*>(base + 2372ull * cap)[idx];
            R.r94 = reinterpret_cast<const float*>(base + 2376ull * cap)[idx];
            R.r100 = reinterpret_cast<const float*>(base + 2380ull * cap)[idx];
            R.r101 = reinterpret_cast<const float*>(base + 2384ull * cap)[idx];
            R.r102 = reinterpret_cast<const float*>(base + 2388ull * cap)[idx];
            R.r103 = reinterpret_cast<const float*>(base + 2392ull * cap)[idx];
            R.r104 = reinterpret_cast<const float*>(base + 2396ull * cap)[idx];
            R.r105 = reinterpret_cast<const float*>(base + 2400ull * cap)[idx];
            R.r117 = reinterpret_cast<const float*>(base + 2404ull * cap)[idx];
            R.r118 = reinterpret_cast<const float*>(base + 2408ull * cap)[idx];
            R.r119 = reinterpret_cast<const float*>(base + 2412ull * cap)[idx];
            R.r127 = reinterpret_cast<const float*>(base + 2416ull * cap)[idx];
            R.r128 = reinterpret_cast<const float*>(base + 2420ull * cap)[idx];
            R.r129 = reinterpret_cast<const float*>(base + 2424ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2428ull * cap)[idx];
        case 24: // roll, context 0
            R.r26 = static_cast<unsigned int>(0);
            R.r7 = reinterpret_cast<const unsigned int*>(base + 2432ull * cap)[idx];
            R.r9 = reinterpret_cast<const unsigned int*>(base + 2436ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 2440ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 2444ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 2448ull * cap)[idx];
            R.r14 = reinterpret_cast<const float*>(base + 2452ull * cap)[idx];
            R.r15 = reinterpret_cast<const float*>(base + 2456ull * cap)[idx];
            R.r16 = reinterpret_cast<const float*>(base + 2460ull * cap)[idx];
            R.r17 = reinterpret_cast<const float*>(base + 2464ull * cap)[idx];
            R.r20 = reinterpret_cast<const unsigned int*>(base + 2468ull * cap)[idx];
            R.r21 = reinterpret_cast<const unsigned int*>(base + 2472ull * cap)[idx];
            R.r22 = reinterpret_cast<const unsigned int*>(base + 2476ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 2480ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 2484ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 2488ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2492ull * cap)[idx];
        case 25: // roll, context 1
            R.r26 = static_cast<unsigned int>(1);
            R.r3 = reinterpret_cast<const float*>(base + 2496ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2500ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 2504ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 2508ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 2512ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 2516ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 2520ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 2524ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 2528ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 2532ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 2536ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 2540ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 2544ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 2548ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 2552ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 2556ull * cap)[idx];
            R.r76 = reinterpret_cast<const float*>(base + 2560ull * cap)[idx];
            R.r77 = reinterpret_cast<const float*>(base + 2564ull * cap)[idx];
            R.r78 = reinterpret_cast<const float*>(base + 2568ull * cap)[idx];
            R.r79 = reinterpret_cast<const unsigned int*>(base + 2572ull * cap)[idx];
            R.r80 = reinterpret_cast<const float*>(base + 2576ull * cap)[idx];
            R.r81 = reinterpret_cast<const float*>(base + 2580ull * cap)[idx];
            R.r82 = reinterpret_cast<const float*>(base + 2584ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 2588ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 2592ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 2596ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2600ull * cap)[idx];
        case 26: // roll, context 2
            R.r26 = static_cast<unsigned int>(2);
            R.r3 = reinterpret_cast<const float*>(base + 2608ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2612ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 2616ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 2620ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 2624ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 2628ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 2632ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 2636ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 2640ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 2644ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 2648ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 2652ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 2656ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 2660ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 2664ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 2668ull * cap)[idx];
            R.r92 = reinterpret_cast<const float*>(base + 2672ull * cap)[idx];
            R.r93 = reinterpret_cast<const float*>(base + 2676ull * cap)[idx];
            R.r94 = reinterpret_cast<const float*>(base + 2680ull * cap)[idx];
            R.r100 = reinterpret_cast<const float*>(base + 2684ull * cap)[idx];
            R.r101 = reinterpret_cast<const float*>(base + 2688ull * cap)[idx];
            R.r102 = reinterpret_cast<const float*>(base + 2692ull * cap)[idx];
            R.r103 = reinterpret_cast<const float*>(base + 2696ull * cap)[idx];
            R.r104 = reinterpret_cast<const float*>(base + 2700ull * cap)[idx];
            R.r105 = reinterpret_cast<const float*>(base + 2704ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2708ull * cap)[idx];
        case 27: // roll, context 3
            R.r26 = static_cast<unsigned int>(3);
            R.r3 = reinterpret_cast<const float*>(base + 2712ull * cap)[idx];
            R.r4 = reinterpret_cast<const float*>(base + 2716ull * cap)[idx];
            R.r5 = reinterpret_cast<const float*>(base + 2720ull * cap)[idx];
            R.r11 = reinterpret_cast<const unsigned int*>(base + 2724ull * cap)[idx];
            R.r12 = reinterpret_cast<const unsigned int*>(base + 2728ull * cap)[idx];
            R.r13 = reinterpret_cast<const unsigned int*>(base + 2732ull * cap)[idx];
            R.r23 = reinterpret_cast<const unsigned int*>(base + 2736ull * cap)[idx];
            R.r24 = reinterpret_cast<const unsigned int*>(base + 2740ull * cap)[idx];
            R.r25 = reinterpret_cast<const unsigned int*>(base + 2744ull * cap)[idx];
            R.r42 = reinterpret_cast<const float*>(base + 2748ull * cap)[idx];
            R.r43 = reinterpret_cast<const float*>(base + 2752ull * cap)[idx];
            R.r44 = reinterpret_cast<const float*>(base + 2756ull * cap)[idx];
            R.r46 = reinterpret_cast<const float*>(base + 2760ull * cap)[idx];
            R.r47 = reinterpret_cast<const float*>(base + 2764ull * cap)[idx];
            R.r48 = reinterpret_cast<const float*>(base + 2768ull * cap)[idx];
            R.r49 = reinterpret_cast<const float*>(base + 2772ull * cap)[idx];
            R.r50 = reinterpret_cast<const float*>(base + 2776ull * cap)[idx];
            R.r51 = reinterpret_cast<const float*>(base + 2780ull * cap)[idx];
            R.r52 = reinterpret_cast<const unsigned int*>(base + 2784ull * cap)[idx];
            R.r83 = reinterpret_cast<const float*>(base + 2788ull * cap)[idx];
            R.r84 = reinterpret_cast<const float*>(base + 2792ull * cap)[idx];
            R.r85 = reinterpret_cast<const float*>(base + 2796ull * cap)[idx];
            R.r87 = reinterpret_cast<const float*>(base + 2800ull * cap)[idx];
            R.r117 = reinterpret_cast<const float*>(base + 2804ull * cap)[idx];
            R.r118 = reinterpret_cast<const float*>(base + 2808ull * cap)[idx];
            R.r119 = reinterpret_cast<const float*>(base + 2812ull * cap)[idx];
            R.r127 = reinterpret_cast<const float*>(base + 2816ull * cap)[idx];
            R.r128 = reinterpret_cast<const float*>(base + 2820ull * cap)[idx];
            R.r129 = reinterpret_cast<const float*>(base + 2824ull * cap)[idx];
            return reinterpret_cast<const unsigned*>(base + 2828ull * cap)[idx];
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
const unsigned long long kQOffs0[] = {0ull, 4ull};
const uint32_t kQRegs1[] = {7u, 9u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 20u, 21u, 22u, 23u, 24u, 25u, 130u, 131u};
const int kQTypes1[] = {LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames1[] = {"w", "h", "k0", "soff", "scnt", "cam0", "cam1", "cam2", "tanf", "smp", "px", "py", "k2", "c0", "c1", "u0", "u1"};
const unsigned long long kQOffs1[] = {16ull, 20ull, 24ull, 28ull, 32ull, 36ull, 40ull, 44ull, 48ull, 52ull, 56ull, 60ull, 64ull, 68ull, 72ull, 76ull, 80ull};
const uint32_t kQRegs2[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u};
const int kQTypes2[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames2[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth"};
const unsigned long long kQOffs2[] = {88ull, 92ull, 96ull, 100ull, 104ull, 108ull, 112ull, 116ull, 120ull, 124ull, 128ull, 132ull, 136ull, 140ull, 144ull, 148ull, 152ull, 156ull, 160ull};
const uint32_t kQRegs3[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 53u, 54u, 55u, 56u};
const int kQTypes3[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames3[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "tmin", "hid", "i", "sp"};
const unsigned long long kQOffs3[] = {168ull, 172ull, 176ull, 180ull, 184ull, 188ull, 192ull, 196ull, 200ull, 204ull, 208ull, 212ull, 216ull, 220ull, 224ull, 228ull, 232ull, 236ull, 240ull, 244ull, 248ull, 252ull, 256ull};
const uint32_t kQRegs4[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 53u, 54u};
const int kQTypes4[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames4[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "tmin", "hid"};
const unsigned long long kQOffs4[] = {264ull, 268ull, 272ull, 276ull, 280ull, 284ull, 288ull, 292ull, 296ull, 300ull, 304ull, 308ull, 312ull, 316ull, 320ull, 324ull, 328ull, 332ull, 336ull, 340ull, 344ull};
const uint32_t kQRegs5[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 53u, 54u};
const int kQTypes5[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames5[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "tmin", "hid"};
const unsigned long long kQOffs5[] = {352ull, 356ull, 360ull, 364ull, 368ull, 372ull, 376ull, 380ull, 384ull, 388ull, 392ull, 396ull, 400ull, 404ull, 408ull, 412ull, 416ull, 420ull, 424ull, 428ull, 432ull};
const uint32_t kQRegs6[] = {3u, 4u, 5u, 49u, 50u, 51u, 76u, 77u, 78u};
const int kQTypes6[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames6[] = {"L0", "L1", "L2", "T0", "T1", "T2", "cr", "cg", "cb"};
const unsigned long long kQOffs6[] = {440ull, 444ull, 448ull, 452ull, 456ull, 460ull, 464ull, 468ull, 472ull};
const uint32_t kQRegs7[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes7[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames7[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs7[] = {480ull, 484ull, 488ull, 492ull, 496ull, 500ull, 504ull, 508ull, 512ull, 516ull, 520ull, 524ull, 528ull, 532ull, 536ull, 540ull, 544ull, 548ull, 552ull, 556ull, 560ull, 564ull, 568ull, 572ull, 576ull, 580ull};
const uint32_t kQRegs8[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes8[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames8[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs8[] = {592ull, 596ull, 600ull, 604ull, 608ull, 612ull, 616ull, 620ull, 624ull, 628ull, 632ull, 636ull, 640ull, 644ull, 648ull, 652ull, 656ull, 660ull, 664ull, 668ull, 672ull, 676ull, 680ull, 684ull, 688ull, 692ull};
const uint32_t kQRegs9[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes9[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames9[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs9[] = {704ull, 708ull, 712ull, 716ull, 720ull, 724ull, 728ull, 732ull, 736ull, 740ull, 744ull, 748ull, 752ull, 756ull, 760ull, 764ull, 768ull, 772ull, 776ull, 780ull, 784ull, 788ull, 792ull, 796ull, 800ull, 804ull};
const uint32_t kQRegs10[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u, 130u};
const int kQTypes10[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames10[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2", "u0"};
const unsigned long long kQOffs10[] = {816ull, 820ull, 824ull, 828ull, 832ull, 836ull, 840ull, 844ull, 848ull, 852ull, 856ull, 860ull, 864ull, 868ull, 872ull, 876ull, 880ull, 884ull, 888ull, 892ull, 896ull, 900ull, 904ull, 908ull, 912ull, 916ull, 920ull};
const uint32_t kQRegs11[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u, 86u};
const int kQTypes11[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames11[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2", "p"};
const unsigned long long kQOffs11[] = {928ull, 932ull, 936ull, 940ull, 944ull, 948ull, 952ull, 956ull, 960ull, 964ull, 968ull, 972ull, 976ull, 980ull, 984ull, 988ull, 992ull, 996ull, 1000ull, 1004ull, 1008ull, 1012ull, 1016ull, 1020ull, 1024ull, 1028ull, 1032ull};
const uint32_t kQRegs12[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes12[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames12[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs12[] = {1040ull, 1044ull, 1048ull, 1052ull, 1056ull, 1060ull, 1064ull, 1068ull, 1072ull, 1076ull, 1080ull, 1084ull, 1088ull, 1092ull, 1096ull, 1100ull, 1104ull, 1108ull, 1112ull, 1116ull, 1120ull, 1124ull, 1128ull, 1132ull, 1136ull, 1140ull};
const uint32_t kQRegs13[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u};
const int kQTypes13[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames13[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn"};
const unsigned long long kQOffs13[] = {1152ull, 1156ull, 1160ull, 1164ull, 1168ull, 1172ull, 1176ull, 1180ull, 1184ull, 1188ull, 1192ull, 1196ull, 1200ull, 1204ull, 1208ull, 1212ull, 1216ull, 1220ull, 1224ull, 1228ull, 1232ull, 1236ull, 1240ull};
const uint32_t kQRegs14[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u};
const int kQTypes14[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames14[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2"};
const unsigned long long kQOffs14[] = {1248ull, 1252ull, 1256ull, 1260ull, 1264ull, 1268ull, 1272ull, 1276ull, 1280ull, 1284ull, 1288ull, 1292ull, 1296ull, 1300ull, 1304ull, 1308ull, 1312ull, 1316ull, 1320ull};
const uint32_t kQRegs15[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u};
const int kQTypes15[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames15[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2"};
const unsigned long long kQOffs15[] = {1328ull, 1332ull, 1336ull, 1340ull, 1344ull, 1348ull, 1352ull, 1356ull, 1360ull, 1364ull, 1368ull, 1372ull, 1376ull, 1380ull, 1384ull, 1388ull, 1392ull, 1396ull, 1400ull, 1404ull, 1408ull, 1412ull, 1416ull, 1420ull, 1424ull};
const uint32_t kQRegs16[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u, 130u, 131u};
const int kQTypes16[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames16[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2", "u0", "u1"};
const unsigned long long kQOffs16[] = {1432ull, 1436ull, 1440ull, 1444ull, 1448ull, 1452ull, 1456ull, 1460ull, 1464ull, 1468ull, 1472ull, 1476ull, 1480ull, 1484ull, 1488ull, 1492ull, 1496ull, 1500ull, 1504ull, 1508ull, 1512ull, 1516ull, 1520ull, 1524ull, 1528ull, 1532ull, 1536ull};
const uint32_t kQRegs17[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u, 106u, 107u, 108u};
const int kQTypes17[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames17[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2", "dx", "dy", "rr2"};
const unsigned long long kQOffs17[] = {1544ull, 1548ull, 1552ull, 1556ull, 1560ull, 1564ull, 1568ull, 1572ull, 1576ull, 1580ull, 1584ull, 1588ull, 1592ull, 1596ull, 1600ull, 1604ull, 1608ull, 1612ull, 1616ull, 1620ull, 1624ull, 1628ull, 1632ull, 1636ull, 1640ull, 1644ull, 1648ull, 1652ull};
const uint32_t kQRegs18[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 88u, 92u, 93u, 94u};
const int kQTypes18[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames18[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "into", "nl0", "nl1", "nl2"};
const unsigned long long kQOffs18[] = {1664ull, 1668ull, 1672ull, 1676ull, 1680ull, 1684ull, 1688ull, 1692ull, 1696ull, 1700ull, 1704ull, 1708ull, 1712ull, 1716ull, 1720ull, 1724ull, 1728ull, 1732ull, 1736ull, 1740ull, 1744ull, 1748ull, 1752ull, 1756ull, 1760ull, 1764ull, 1768ull};
const uint32_t kQRegs19[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 88u, 111u, 112u, 113u};
const int kQTypes19[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames19[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "into", "nnt", "ddn", "c2"};
const unsigned long long kQOffs19[] = {1776ull, 1780ull, 1784ull, 1788ull, 1792ull, 1796ull, 1800ull, 1804ull, 1808ull, 1812ull, 1816ull, 1820ull, 1824ull, 1828ull, 1832ull, 1836ull, 1840ull, 1844ull, 1848ull, 1852ull, 1856ull, 1860ull, 1864ull, 1868ull, 1872ull, 1876ull, 1880ull};
const uint32_t kQRegs20[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 117u, 118u, 119u, 127u, 128u, 129u, 130u};
const int kQTypes20[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32};
const char* const kQNames20[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "td0", "td1", "td2", "pp", "rp", "tp", "u0"};
const unsigned long long kQOffs20[] = {1888ull, 1892ull, 1896ull, 1900ull, 1904ull, 1908ull, 1912ull, 1916ull, 1920ull, 1924ull, 1928ull, 1932ull, 1936ull, 1940ull, 1944ull, 1948ull, 1952ull, 1956ull, 1960ull, 1964ull, 1968ull, 1972ull, 1976ull, 1980ull, 1984ull, 1988ull, 1992ull, 1996ull, 2000ull, 2004ull};
const uint32_t kQRegs21[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 128u};
const int kQTypes21[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames21[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "rp"};
const unsigned long long kQOffs21[] = {2016ull, 2020ull, 2024ull, 2028ull, 2032ull, 2036ull, 2040ull, 2044ull, 2048ull, 2052ull, 2056ull, 2060ull, 2064ull, 2068ull, 2072ull, 2076ull, 2080ull, 2084ull, 2088ull, 2092ull, 2096ull, 2100ull, 2104ull, 2108ull};
const uint32_t kQRegs22[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 117u, 118u, 119u, 129u};
const int kQTypes22[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames22[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "td0", "td1", "td2", "tp"};
const unsigned long long kQOffs22[] = {2120ull, 2124ull, 2128ull, 2132ull, 2136ull, 2140ull, 2144ull, 2148ull, 2152ull, 2156ull, 2160ull, 2164ull, 2168ull, 2172ull, 2176ull, 2180ull, 2184ull, 2188ull, 2192ull, 2196ull};
const uint32_t kQRegs23[] = {3u, 4u, 5u, 7u, 9u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 20u, 21u, 22u, 23u, 24u, 25u, 26u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u, 87u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u, 117u, 118u, 119u, 127u, 128u, 129u};
const int kQTypes23[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames23[] = {"L0", "L1", "L2", "w", "h", "k0", "soff", "scnt", "cam0", "cam1", "cam2", "tanf", "smp", "px", "py", "k2", "c0", "c1", "rpt", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2", "dn", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2", "td0", "td1", "td2", "pp", "rp", "tp"};
const unsigned long long kQOffs23[] = {2208ull, 2212ull, 2216ull, 2220ull, 2224ull, 2228ull, 2232ull, 2236ull, 2240ull, 2244ull, 2248ull, 2252ull, 2256ull, 2260ull, 2264ull, 2268ull, 2272ull, 2276ull, 2280ull, 2284ull, 2288ull, 2292ull, 2296ull, 2300ull, 2304ull, 2308ull, 2312ull, 2316ull, 2320ull, 2324ull, 2328ull, 2332ull, 2336ull, 2340ull, 2344ull, 2348ull, 2352ull, 2356ull, 2360ull, 2364ull, 2368ull, 2372ull, 2376ull, 2380ull, 2384ull, 2388ull, 2392ull, 2396ull, 2400ull, 2404ull, 2408ull, 2412ull, 2416ull, 2420ull, 2424ull};
const uint32_t kQRegs24[] = {7u, 9u, 11u, 12u, 13u, 14u, 15u, 16u, 17u, 20u, 21u, 22u, 23u, 24u, 25u};
const int kQTypes24[] = {LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32};
const char* const kQNames24[] = {"w", "h", "k0", "soff", "scnt", "cam0", "cam1", "cam2", "tanf", "smp", "px", "py", "k2", "c0", "c1"};
const unsigned long long kQOffs24[] = {2432ull, 2436ull, 2440ull, 2444ull, 2448ull, 2452ull, 2456ull, 2460ull, 2464ull, 2468ull, 2472ull, 2476ull, 2480ull, 2484ull, 2488ull};
const uint32_t kQRegs25[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 49u, 50u, 51u, 52u, 76u, 77u, 78u, 79u, 80u, 81u, 82u, 83u, 84u, 85u};
const int kQTypes25[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames25[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "T0", "T1", "T2", "depth", "cr", "cg", "cb", "mat", "x0", "x1", "x2", "n0", "n1", "n2"};
const unsigned long long kQOffs25[] = {2496ull, 2500ull, 2504ull, 2508ull, 2512ull, 2516ull, 2520ull, 2524ull, 2528ull, 2532ull, 2536ull, 2540ull, 2544ull, 2548ull, 2552ull, 2556ull, 2560ull, 2564ull, 2568ull, 2572ull, 2576ull, 2580ull, 2584ull, 2588ull, 2592ull, 2596ull};
const uint32_t kQRegs26[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 92u, 93u, 94u, 100u, 101u, 102u, 103u, 104u, 105u};
const int kQTypes26[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames26[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "nl0", "nl1", "nl2", "uu0", "uu1", "uu2", "vv0", "vv1", "vv2"};
const unsigned long long kQOffs26[] = {2608ull, 2612ull, 2616ull, 2620ull, 2624ull, 2628ull, 2632ull, 2636ull, 2640ull, 2644ull, 2648ull, 2652ull, 2656ull, 2660ull, 2664ull, 2668ull, 2672ull, 2676ull, 2680ull, 2684ull, 2688ull, 2692ull, 2696ull, 2700ull, 2704ull};
const uint32_t kQRegs27[] = {3u, 4u, 5u, 11u, 12u, 13u, 23u, 24u, 25u, 42u, 43u, 44u, 46u, 47u, 48u, 49u, 50u, 51u, 52u, 83u, 84u, 85u, 87u, 117u, 118u, 119u, 127u, 128u, 129u};
const int kQTypes27[] = {LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_U32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32, LOOM_B200_F32};
const char* const kQNames27[] = {"L0", "L1", "L2", "k0", "soff", "scnt", "k2", "c0", "c1", "d0", "d1", "d2", "o0", "o1", "o2", "T0", "T1", "T2", "depth", "n0", "n1", "n2", "dn", "td0", "td1", "td2", "pp", "rp", "tp"};
const unsigned long long kQOffs27[] = {2712ull, 2716ull, 2720ull, 2724ull, 2728ull, 2732ull, 2736ull, 2740ull, 2744ull, 2748ull, 2752ull, 2756ull, 2760ull, 2764ull, 2768ull, 2772ull, 2776ull, 2780ull, 2784ull, 2788ull, 2792ull, 2796ull, 2800ull, 2804ull, 2808ull, 2812ull, 2816ull, 2820ull, 2824ull};
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
    {kQOffs0, 8ull},
    {kQOffs1, 84ull},
    {kQOffs2, 164ull},
    {kQOffs3, 260ull},
    {kQOffs4, 348ull},
    {kQOffs5, 436ull},
    {kQOffs6, 476ull},
    {kQOffs7, 584ull},
    {kQOffs8, 696ull},
    {kQOffs9, 808ull},
    {kQOffs10, 924ull},
    {kQOffs11, 1036ull},
    {kQOffs12, 1144ull},
    {kQOffs13, 1244ull},
    {kQOffs14, 1324ull},
    {kQOffs15, 1428ull},
    {kQOffs16, 1540ull},
    {kQOffs17, 1656ull},
    {kQOffs18, 1772ull},
    {kQOffs19, 1884ull},
    {kQOffs20, 2008ull},
    {kQOffs21, 2112ull},
    {kQOffs22, 2200ull},
    {kQOffs23, 2428ull},
    {kQOffs24, 2492ull},
    {kQOffs25, 2600ull},
    {kQOffs26, 2708ull},
    {kQOffs27, 2828ull},
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

} } // namespace loom_b200::k_sphere_pt_f32

extern const loom_b200::KernelEntry loom_b200_entry_sphere_pt_f32;
const loom_b200::KernelEntry loom_b200_entry_sphere_pt_f32 = {
    &loom_b200::k_sphere_pt_f32::kInfo, loom_b200::k_sphere_pt_f32::K::kRowBytes, 28,
    &loom_b200::k_sphere_pt_f32::launch_plain, &loom_b200::k_sphere_pt_f32::launch_regroup,
    &loom_b200::k_sphere_pt_f32::regroup_occupancy,
    loom_b200::k_sphere_pt_f32::kQueues, loom_b200::k_sphere_pt_f32::kSegments,
    loom_b200::k_sphere_pt_f32::kRegCaps, 8u};
