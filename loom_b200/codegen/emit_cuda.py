"""Lower a Loom kernel (text IR) to CUDA C++ for the B200 engines.

For every kernel the generator writes one translation unit that defines a
struct ``K`` with

* ``Regs``            the Loom register file as scalars (kept in CUDA
                      registers); Union registers (Loom src/common/union.hpp)
                      are stored as unsigned integers and bit-cast per view;
* ``run_burst<kProf>`` the whole program as a goto CFG that can be entered at
                      any block and stops after a budget of blocks: the
                      plain engine runs it from block 0 with the step guard
                      as budget, the regrouping engine runs bursts of a few
                      blocks between warp votes;
* ``save/restore(b)`` the live-in registers of block b to/from the queue of
                      block b (an SoA segment per block and round parity);
* ``load_inputs`` / ``store_outputs`` the input/output columns;

plus the host-side descriptor and launchers.  Op semantics follow Loom
src/vm/operators.hpp and the std:: functors exactly as standard_eval applies
them (core.hpp:740-750): arguments are converted to the functor's operand
type, the functor's result type is kept (T for arithmetic, bool for
comparisons and logic), and the result is converted to the destination
variable's type.  The TU is compiled with -fmad=false and IEEE division and
square root so that float arithmetic rounds like the scalar backend.
"""

from __future__ import annotations

import math
import struct
from typing import Dict, List

from .ir import (
    FLOAT_TYPES,
    HALT,
    INT_TYPES,
    TYPE_BYTES,
    Compute,
    Jump,
    Kernel,
    Operand,
    ParmJump,
)


# Register cap of the regrouping megakernel.  The persistent kernel keeps
# every lane busy from one resident warp set, so latency is hidden only by
# the warps an SM holds: 64 registers fit 2 CTAs of 512 threads (32 warps)
# per SM, against 16 warps at the compiler's own choice of 128 for the
# sphere path tracer.  The spills this costs stay in L1; measured on one
# B200, 1024x768x64 sphere path tracer 41.0 ms vs 52.5 ms, 256 batched
# render requests 156.6 ms vs 180.4 ms, outputs identical.
REGROUP_MAX_REGS = 64

# Further register caps compiled for kernels large enough to reach the cap
# (more static instructions than REG_VARIANT_MIN_INSTR): the tuner picks one
# per workload (opts.max_regs), trading warps per SM against spills.
REG_VARIANTS = (32, 40, 48, 56, 80, 96, 128)
REG_VARIANT_MIN_INSTR = 300
# Small kernels: the megakernel's own state dominates their registers, and a
# cap that fits one more CTA per SM can pay for latency-bound loops.
SMALL_REG_VARIANTS = (40, 48)

# Long blocks: at least this many instructions.  The software-stepped
# schedule can hold lanes that reach one back until enough of the warp's
# lanes stand there (opts.defer_lanes), so that its long code runs at a
# higher lane efficiency (the path tracers' random-number subroutine).
LONG_BLOCK_INSTR = 96


def long_blocks(k: Kernel) -> List[int]:
    """Blocks of at least LONG_BLOCK_INSTR instructions, longest first (at
    most 4)."""
    counts = k.instr_counts()
    return sorted((b for b in range(k.num_blocks) if counts[b] >= LONG_BLOCK_INSTR), key=lambda b: -counts[b])[:4]


def reg_caps(k: Kernel) -> List[int]:
    """Register caps of the megakernel compiled for `k`, default first."""
    extra = REG_VARIANTS if sum(k.instr_counts()) > REG_VARIANT_MIN_INSTR else SMALL_REG_VARIANTS
    return [REGROUP_MAX_REGS] + [c for c in extra if c != REGROUP_MAX_REGS]


CTYPE = {
    "b8": "bool",
    "i8": "signed char",
    "u8": "unsigned char",
    "i16": "short",
    "u16": "unsigned short",
    "i32": "int",
    "u32": "unsigned int",
    "i64": "long long",
    "u64": "unsigned long long",
    "f32": "float",
    "f64": "double",
}

ABI_TYPE = {
    "b8": "LOOM_B200_B8",
    "i8": "LOOM_B200_I8",
    "u8": "LOOM_B200_U8",
    "i16": "LOOM_B200_I16",
    "u16": "LOOM_B200_U16",
    "i32": "LOOM_B200_I32",
    "u32": "LOOM_B200_U32",
    "i64": "LOOM_B200_I64",
    "u64": "LOOM_B200_U64",
    "f32": "LOOM_B200_F32",
    "f64": "LOOM_B200_F64",
}

CMP = {"eq": "==", "ne": "!=", "gt": ">", "lt": "<", "ge": ">=", "le": "<="}
ARITH = {"add": "+", "sub": "-", "mul": "*", "div": "/", "mod": "%"}
BITS = {"band": "&", "bor": "|", "bxor": "^", "shl": "<<", "shr": ">>"}
LOGIC = {"land": "&&", "lor": "||"}
UNARY_FN = {
    "round": "op_round",
    "ceil": "op_ceil",
    "floor": "op_floor",
    "trunc": "op_trunc",
    "sqrt": "op_sqrt",
    "sin": "op_sin",
    "cos": "op_cos",
    "rsqrt": "op_rsqrt",
}


def literal(op: Operand) -> str:
    """Exact C++ spelling of a literal's bit pattern."""
    t = op.type
    ct = CTYPE[t]
    if t == "f32":
        v = struct.unpack("<f", struct.pack("<I", op.bits & 0xFFFFFFFF))[0]
        if math.isfinite(v):
            return f"({v.hex()}f)"
        return f"__uint_as_float({op.bits & 0xFFFFFFFF:#x}u)"
    if t == "f64":
        v = struct.unpack("<d", struct.pack("<Q", op.bits))[0]
        if math.isfinite(v):
            return f"({v.hex()})"
        return f"__longlong_as_double({op.bits:#x}ll)"
    if t == "b8":
        return "true" if op.bits & 1 else "false"
    nbits = TYPE_BYTES[t] * 8
    bits = op.bits & ((1 << nbits) - 1)
    return f"(({ct}){bits:#x}ull)"


class Lowering:
    def __init__(self, k: Kernel):
        self.k = k
        self.pc = k.pc_reg()
        self.regs = {r.idx: r for r in k.regs}

    # ------------------------------------------------------------ views
    def rname(self, idx: int) -> str:
        return f"R.r{idx}"

    def read(self, op: Operand) -> str:
        if op.is_literal:
            return literal(op)
        reg = self.regs[op.reg]
        if reg.storage == op.type:
            return self.rname(op.reg)
        return f"bitcast<{CTYPE[op.type]}>({self.rname(op.reg)})"

    def write(self, dst: Operand, expr: str) -> str:
        reg = self.regs[dst.reg]
        val = f"static_cast<{CTYPE[dst.type]}>({expr})"
        if reg.storage == dst.type:
            return f"{self.rname(dst.reg)} = {val};"
        return f"{self.rname(dst.reg)} = bitcast<{CTYPE[reg.storage]}>({val});"

    # ------------------------------------------------------------ ops
    def expr(self, ins: Compute) -> str:
        op = ins.op
        a = [self.read(x) for x in ins.args]
        ot = ins.optype

        def cv(i: int, t: str) -> str:
            return f"static_cast<{CTYPE[t]}>({a[i]})"

        if op == "mov":
            return a[0]
        if op == "cmov":
            return f"(({a[0]}) ? ({a[1]}) : ({a[2]}))"
        if op in ("fma", "fms"):
            t = ins.args[0].type
            z = a[2] if op == "fma" else f"(-({a[2]}))"
            return f"op_fma({a[0]}, {a[1]}, {z})"
        if op == "assert_fp":
            return f"op_assert_fp({a[0]}, ctx)"
        if op == "tab":
            (t,) = ot
            return f"table_load<{CTYPE[t]}>(*ctx.cols, static_cast<unsigned>({a[0]}))"
        if op == "sct":
            t, _ = ot
            consts = [literal(c) for c in ins.consts]
            idx = a[0]
            e = consts[-1]
            for i in reversed(range(len(consts) - 1)):
                e = f"(({idx}) == {i} ? {consts[i]} : {e})"
            return f"static_cast<{CTYPE[t]}>({e})"
        if op == "slt":
            t, _ = ot
            idx = a[0]
            vals = a[1:]
            e = f"static_cast<{CTYPE[t]}>({vals[-1]})"
            for i in reversed(range(len(vals) - 1)):
                e = f"(({idx}) == {i} ? static_cast<{CTYPE[t]}>({vals[i]}) : {e})"
            return e
        if op == "pacc":
            t, it, acc, cmp = ot
            c = f"static_cast<{CTYPE[it]}>({cv(1, t)} {CMP[cmp]} {cv(2, t)})"
            return f"static_cast<{CTYPE[it]}>({cv(0, it)} {LOGIC[acc]} {c})"
        (t,) = ot
        ct = CTYPE[t]
        if op in ARITH:
            return f"static_cast<{ct}>({cv(0, t)} {ARITH[op]} {cv(1, t)})"
        if op in BITS:
            return f"static_cast<{ct}>({cv(0, t)} {BITS[op]} {cv(1, t)})"
        if op in CMP:
            return f"static_cast<bool>({cv(0, t)} {CMP[op]} {cv(1, t)})"
        if op in LOGIC:
            return f"static_cast<bool>({cv(0, t)} {LOGIC[op]} {cv(1, t)})"
        if op == "lnot":
            return f"static_cast<bool>(!{cv(0, t)})"
        if op == "neg":
            return f"static_cast<{ct}>(-{cv(0, t)})"
        if op == "bnot":
            return f"static_cast<{ct}>(~{cv(0, t)})"
        if op == "abs":
            if t in FLOAT_TYPES:
                return f"op_abs({cv(0, t)})"
            if t.startswith("u"):
                return cv(0, t)
            wide = "long long" if t == "i64" else "int"
            return f"static_cast<{ct}>(op_abs(static_cast<{wide}>({cv(0, t)})))"
        if op == "max":
            return f"op_max<{ct}>({cv(0, t)}, {cv(1, t)})"
        if op == "min":
            return f"op_min<{ct}>({cv(0, t)}, {cv(1, t)})"
        if op == "copysign":
            return f"op_copysign({cv(0, t)}, {cv(1, t)})"
        if op in UNARY_FN:
            return f"{UNARY_FN[op]}({cv(0, t)})"
        raise NotImplementedError(f"{self.k.name}: op {op}")

    def body(self, instrs, indent: str) -> List[str]:
        out = []
        for ins in instrs:
            if isinstance(ins, Compute):
                out.append(indent + self.write(ins.dst, self.expr(ins)))
        return out

    # ------------------------------------------------------------ transfers
    def next_expr(self, blk) -> str:
        """C++ expression of the next block index (kHalt for HALT)."""
        t = blk.terminator
        if t is None:
            return "kHalt"
        if isinstance(t, Jump):
            return self.target(t.target)
        v = self.read(t.var)
        tg = [self.target(x) for x in t.targets]
        if len(tg) == 2:
            # Loom's scalar dispatch: any non-zero selects the second label
            # (bse.hpp:180-185).
            return f"(({v}) ? {tg[1]} : {tg[0]})"
        e = "kHalt"  # out-of-table values leave the thread where it is
        for i in reversed(range(len(tg))):
            e = f"(({v}) == {i} ? {tg[i]} : {e})"
        return e

    @staticmethod
    def target(t: int) -> str:
        return "kHalt" if t == HALT else str(t)

    def goto_transfer(self, blk, indent: str) -> List[str]:
        t = blk.terminator
        if t is None:
            return [indent + "goto L_HALT;"]
        if isinstance(t, Jump):
            return [indent + f"goto {self.label(t.target)};"]
        v = self.read(t.var)
        if len(t.targets) == 2:
            return [
                indent
                + f"if({v}) goto {self.label(t.targets[1])}; else goto {self.label(t.targets[0])};"
            ]
        lines = [indent + f"switch({v}) {{"]
        for i, tg in enumerate(t.targets):
            lines.append(indent + f"case {i}: goto {self.label(tg)};")
        lines.append(indent + "default: goto L_HALT;")
        lines.append(indent + "}")
        return lines

    @staticmethod
    def label(t: int) -> str:
        return "L_HALT" if t == HALT else f"L_B{t}"


def pack_slots(items, start: int) -> Dict:
    """Queue row layout from `start` (bytes per entry): items (register,
    bytes) and the input index ("tid", 4).  Registers of 8 and 4 bytes and
    the index are packed largest first into slots of 16 bytes, each at an
    offset that is a multiple of its size; the last slot shrinks to 8 or 4
    bytes when that holds its contents; registers of 1 or 2 bytes get a slot
    each.  Returns {"slots": [(off, width, [(item, sub)])], "cols": {reg: (off,
    sub, width)}, "tid": (off, sub, width), "end": next offset, a multiple
    of 8}."""
    wide = sorted([(r, n) for r, n in items if n >= 4], key=lambda x: (-x[1], x[0])) + [("tid", 4)]
    narrow = sorted([(r, n) for r, n in items if n < 4], key=lambda x: (-x[1], x[0]))
    slots = []
    cur, used = [], 0
    for it, n in wide:
        if used + n > 16:
            slots.append((cur, used))
            cur, used = [], 0
        cur.append((it, used, n))
        used += n
    if cur:
        slots.append((cur, used))
    out, off = [], start
    for contents, used in slots:
        width = 16 if used > 8 else (8 if used > 4 else 4)
        out.append((off, width, [(it, sub) for it, sub, _ in contents]))
        off += width
    for it, n in narrow:
        out.append((off, n, [(it, 0)]))
        off += n
    end = (off + 7) // 8 * 8
    cols, tid = {}, None
    for o, wdt, contents in out:
        for it, sub in contents:
            if it == "tid":
                tid = (o, sub, wdt)
            else:
                cols[it] = (o, sub, wdt)
    return {"slots": out, "cols": cols, "tid": tid, "end": end}


def generate(k: Kernel) -> str:
    L = Lowering(k)
    name = k.name
    nb = k.num_blocks
    nin = len(k.inputs)
    nout = len(k.outputs)
    live_in, _ = k.liveness()
    state = k.state_regs()
    counts = k.instr_counts()
    live_bytes = [sum(L.regs[r].nbytes for r in li) for li in live_in]
    regs = [r for r in k.regs if r.idx != L.pc]
    if nin + nout > 96:
        raise ValueError(f"{name}: too many columns")
    # work queues: one per block plus one per context of each dispatch block
    queues = k.queues()
    qlive = k.queue_liveness()
    disp = k.dispatch_blocks()
    nq = len(queues)
    qbytes = [sum(L.regs[r].nbytes for r in li) for li in qlive]
    # queue segments: per queue, the live-in registers and the u32 input
    # index packed into slots of 16 bytes per entry (then 8, 4: the rest),
    # so a lane saves or restores four 32-bit values with one 128-bit access
    # and a warp's 32 entries of a slot are 512 contiguous bytes; registers
    # of 1 or 2 bytes keep slots of their own
    layout = []
    row_total = 0
    for q in range(nq):
        layout.append(pack_slots([(r, L.regs[r].nbytes) for r in qlive[q]], row_total))
        row_total = layout[-1]["end"]

    o: List[str] = []
    w = o.append
    w(f"// Generated by loom_b200.codegen from loom_b200/ir/{name}.lir.")
    w(f"// Kernel IR digest {k.digest()}; regenerate instead of editing.")
    w('#include "../engine/plain.cuh"')
    w('#include "../engine/regroup.cuh"')
    w('#include "../runtime_iface.h"')
    w("")
    w(f"namespace loom_b200 {{ namespace k_{name} {{")
    w("")
    w(f"__constant__ unsigned kInstrTab[{nb}] = {{{', '.join(map(str, counts))}}};")
    w(f"__constant__ unsigned kLiveTab[{nq}] = {{{', '.join(map(str, qbytes))}}};")
    w(f"__constant__ int kQueueBlock[{nq}] = {{{', '.join(str(b) for b, _ in queues)}}};")
    # Regrouping cost model: a group of g lanes at block b either runs it
    # now (I_b warp instructions) or parks (C_b column stores now, C_b loads
    # per restored tile of 32, then I_b at full width); parking is cheaper
    # while g < 32 (I_b - C_b) / (I_b + C_b), which is the block's quorum.
    quorum = []
    for b in range(nb):
        cols = max((len(qlive[q]) for q, (qb, _) in enumerate(queues) if qb == b), default=0) + 1
        ib = counts[b]
        quorum.append(min(28, max(0, math.ceil(32 * (ib - cols) / (ib + cols)))) if ib > cols else 0)
    heavy = {b for b in range(nb) if quorum[b] > 0}
    w(f"__constant__ unsigned kQuorumTab[{nb}] = {{{', '.join(map(str, quorum))}}};")
    w(f"__constant__ unsigned kRankTab[{nb}] = {{{', '.join(map(str, k.rpo_ranks()))}}};")
    w("")
    w("struct K")
    w("{")
    w(f"    static constexpr int kNumBlocks = {nb};")
    w(f"    static constexpr int kNumQueues = {nq};")
    w(f"    static constexpr int kRegroupMaxRegs = {REGROUP_MAX_REGS};")
    # small kernels: two inlined copies of their code in the megakernel
    w(f"    static constexpr bool kSplitCallSites = {'true' if sum(counts) <= REG_VARIANT_MIN_INSTR else 'false'};")
    w("    struct Regs")
    w("    {")
    for r in regs:
        w(f"        {CTYPE[r.storage]} r{r.idx}; // {r.name}: {','.join(r.types)}")
    if not regs:
        w("        int unused;")
    w("    };")
    w("")
    # ---- inputs / outputs
    w("    struct In")
    w("    {")
    for i, (reg, t, vname) in enumerate(k.inputs):
        w(f"        {CTYPE[t]} v{i}; // {vname}")
    if not k.inputs:
        w("        int unused;")
    w("    };")
    w("")
    w("    // Reads the input columns of thread `tid` (a NULL column is iota).")
    w("    __device__ __forceinline__ static void")
    w("    load_in(In& in, const Columns& c, const unsigned long long tid)")
    w("    {")
    for i, (reg, t, vname) in enumerate(k.inputs):
        w(f"        in.v{i} = load_input<{CTYPE[t]}>(c, {i}, tid);")
    w("        (void)in; (void)c; (void)tid;")
    w("    }")
    w("")
    w("    // Loom's set_inputs: input variables written, every other register zero.")
    w("    // Only registers live at START (those its queue carries) are written:")
    w("    // the others are written before they are read on every path.")
    w("    __device__ __forceinline__ static void")
    w("    start(Regs& R, const In& in)")
    w("    {")
    live0 = qlive[queues.index((0, None))] if k.blocks else set()
    in_regs = {reg for reg, _, _ in k.inputs}
    for r in regs:
        if r.idx in live0 and r.idx not in in_regs:
            w(f"        R.r{r.idx} = 0;")
    for i, (reg, t, vname) in enumerate(k.inputs):
        w("        " + L.write(Operand(type=t, reg=reg), f"in.v{i}"))
    w("        (void)in;")
    w("    }")
    w("")
    w("    __device__ __forceinline__ static void")
    w("    load_inputs(Regs& R, const Columns& c, const unsigned long long tid)")
    w("    {")
    w("        In in;")
    w("        load_in(in, c, tid);")
    w("        start(R, in);")
    w("    }")
    w("")
    w("    __device__ __forceinline__ static void")
    w("    store_outputs(const Regs& R, const Columns& c, const unsigned long long tid)")
    w("    {")
    for j, (reg, t, vname) in enumerate(k.outputs):
        ct = CTYPE[t]
        w(f"        static_cast<{ct}*>(c.p[{nin + j}])[col_index(c, tid)] = {L.read(Operand(type=t, reg=reg))}; // {vname}")
    w("    }")
    w("")
    w("    __device__ __forceinline__ static unsigned instr(const int b) { return kInstrTab[b]; }")
    w("    __device__ __forceinline__ static unsigned live_bytes(const int q) { return kLiveTab[q]; }")
    w("    __device__ __forceinline__ static int block_of(const int q) { return kQueueBlock[q]; }")
    w("    __device__ __forceinline__ static unsigned quorum(const int b) { return kQuorumTab[b]; }")
    w("    __device__ __forceinline__ static unsigned rank(const int b) { return kRankTab[b]; }")
    lb = long_blocks(k)
    w(f"    static constexpr int kNumLong = {len(lb)};")
    w("    // j-th long block (most instructions first)")
    w("    __device__ __forceinline__ static int long_block(const int j)")
    w("    {")
    if lb:
        w("        switch(j)")
        w("        {")
        for j, b in enumerate(lb):
            w(f"        case {j}: return {b};")
        w("        default: return -1;")
        w("        }")
    else:
        w("        (void)j;")
        w("        return -1;")
    w("    }")
    w("")
    per_block = [[qi for qi, (b, _) in enumerate(queues) if b == blk] for blk in range(nb)]
    maxq = max(len(x) for x in per_block)
    w(f"    static constexpr int kMaxQueuesPerBlock = {maxq};")
    w("    // j-th queue holding threads that stand at block b (-1: none).")
    w("    __device__ __forceinline__ static int")
    w("    queue_list(const int b, const int j)")
    w("    {")
    multi = [(blk, ql) for blk, ql in enumerate(per_block) if len(ql) > 1]
    for blk, ql in multi:
        w(f"        if(b == {blk})")
        w("        {")
        w("            switch(j)")
        w("            {")
        for j, qi in enumerate(ql):
            w(f"            case {j}: return {qi};")
        w("            default: return -1;")
        w("            }")
        w("        }")
    w("        return j == 0 ? b : -1;")
    w("    }")
    w("")
    w("    // Queue a thread standing at block pc waits in: the block's own queue,")
    w("    // or for a dispatch block the queue of the context its register selects.")
    w("    __device__ __forceinline__ static int")
    w("    queue_of(const int pc, const Regs& R)")
    w("    {")
    w("        (void)R;")
    for d, (v, ctx) in sorted(disp.items()):
        w(f"        if(pc == {d})")
        w("        {")
        w(f"            switch(static_cast<unsigned long long>(R.r{v}))")
        w("            {")
        for kk in ctx:
            w(f"            case {kk}ull: return {queues.index((d, kk))};")
        w("            default: break;")
        w("            }")
        w("        }")
    w("        return pc;")
    w("    }")
    w("")
    # ---- run_burst (goto CFG entered at any block, bounded by a budget)
    # the budget is counted at loop headers only (targets of edges that go
    # back in reverse post-order): every cycle passes one, and the blocks in
    # between have no early exit, so a diverged warp reconverges at their
    # post-dominators as in straight CUDA
    rank = k.rpo_ranks()
    headers = {t for b in k.blocks for t in b.successors() if t != HALT and rank[t] <= rank[b.idx]}
    w("    // Runs the lane's own path from block `entry` for at most `budget`")
    w("    // loop iterations (visits of a loop header); returns the block it")
    w("    // stopped at, or kHalt.  With `stop_heavy`, a block whose quorum is")
    w("    // above zero is entered only as the first block of the burst, when")
    w("    // the warp's vote chose it.  A block that loops on itself takes up")
    w("    // to `spin` further iterations without spending budget (a loop the")
    w("    // warp's lanes run together needs no step of its own per iteration).")
    w("    template <bool kProf>")
    w("    __device__ __forceinline__ static int")
    w("    run_burst(const int entry, Regs& R, Ctx& ctx, unsigned budget, const bool stop_heavy = false,")
    w("              unsigned spin = 0u)")
    w("    {")
    w("        (void)ctx;")
    w("        (void)stop_heavy;")
    w("        (void)spin;")
    w("        bool fresh = true; // no block run yet in this burst")
    w("        (void)fresh;")
    w("        switch(entry)")
    w("        {")
    for blk in k.blocks:
        w(f"        case {blk.idx}: goto L_B{blk.idx};")
    w("        default: return kHalt;")
    w("        }")
    for blk in k.blocks:
        w(f"    L_B{blk.idx}: // {blk.label}")
        transfer = L.goto_transfer(blk, "        ")
        own = f"goto L_B{blk.idx};"
        self_loop = blk.idx in headers and blk.idx in blk.successors()
        if blk.idx in heavy or self_loop:
            # a lane that loops on the block keeps going; one that comes
            # from another block waits for the warp's vote
            if blk.idx in heavy:
                w(f"        if(stop_heavy && !fresh) return {blk.idx};")
            w(f"    L_B{blk.idx}_again:")
            back = f"goto L_B{blk.idx}_again;"
            if self_loop:
                back = f"{{ if(spin != 0u) {{ --spin; goto L_B{blk.idx}_spin; }} goto L_B{blk.idx}_again; }}"
            transfer = [t.replace(own, back) for t in transfer]
        if blk.idx in headers:
            w(f"        if(budget == 0u) return {blk.idx};")
            w("        --budget;")
        if self_loop:
            w(f"    L_B{blk.idx}_spin:")
        if heavy:
            w("        fresh = false;")
        w(f"        if constexpr(kProf) count_block(ctx, {blk.idx}, {len(blk.instrs)}u);")
        o.extend(L.body(blk.instrs, "        "))
        o.extend(transfer)
    w("    L_HALT:")
    w("        return kHalt;")
    w("    }")
    w("")
    # ---- save / restore: queue (parity, block) holds the block's live-in
    # registers and the input index, one SoA column each
    w(f"    static constexpr unsigned long long kRowBytes = {row_total}ull;")
    for fn in ("save", "restore"):
        w("    __device__ __forceinline__ static " + ("void" if fn == "save" else "unsigned"))
        if fn == "save":
            w("    save(const int q, const Regs& R, char* st, const unsigned cap, const unsigned par,")
            w("         const unsigned idx, const unsigned tid)")
        else:
            w("    restore(const int q, Regs& R, const char* st, const unsigned cap, const unsigned par,")
            w("            const unsigned idx)")
        w("    {")
        q = "" if fn == "save" else "const "
        w(f"        {q}char* base = st + static_cast<unsigned long long>(par) * kRowBytes * cap;")
        w("        switch(q)")
        w("        {")
        for qi, (b, kk) in enumerate(queues):
            w(f"        case {qi}: // {k.blocks[b].label}" + ("" if kk is None else f", context {kk}"))
            w("        {")
            if fn == "restore" and kk is not None:
                v = disp[b][0]
                w(f"            R.r{v} = static_cast<{CTYPE[L.regs[v].storage]}>({kk});")
            tid_expr = None
            for si, (off, wdt, contents) in enumerate(layout[qi]["slots"]):
                vt = {16: "uint4", 8: "uint2", 4: "unsigned", 2: "unsigned short", 1: "unsigned char"}[wdt]
                slot = f"reinterpret_cast<{q}{vt}*>(base + {off}ull * cap)[idx]"
                if wdt <= 2:
                    # a narrow register alone in its slot
                    (r, _), = contents
                    stt = CTYPE[L.regs[r].storage]
                    if fn == "save":
                        w(f"            {slot} = bitcast<{vt}>(R.r{r});")
                    else:
                        w(f"            R.r{r} = bitcast<{stt}>({slot});")
                    continue
                words = ["x", "y", "z", "w"][: wdt // 4] if wdt > 4 else [None]
                def word(sub):
                    return f"v{si}" if words == [None] else f"v{si}.{words[sub // 4]}"
                if fn == "save":
                    w(f"            {{")
                    w(f"                {vt} v{si};")
                    for it, sub in contents:
                        if it == "tid":
                            w(f"                {word(sub)} = tid;")
                        elif L.regs[it].nbytes == 8:
                            w(f"                {{ const unsigned long long b = bitcast<unsigned long long>(R.r{it});")
                            w(f"                  {word(sub)} = static_cast<unsigned>(b); {word(sub + 4)} = static_cast<unsigned>(b >> 32); }}")
                        else:
                            w(f"                {word(sub)} = bitcast<unsigned>(R.r{it});")
                    w(f"                {slot} = v{si};")
                    w(f"            }}")
                else:
                    w(f"            const {vt} v{si} = {slot};")
                    for it, sub in contents:
                        if it == "tid":
                            tid_expr = word(sub)
                        elif L.regs[it].nbytes == 8:
                            stt = CTYPE[L.regs[it].storage]
                            w(f"            R.r{it} = bitcast<{stt}>((static_cast<unsigned long long>({word(sub + 4)}) << 32) | {word(sub)});")
                        else:
                            stt = CTYPE[L.regs[it].storage]
                            w(f"            R.r{it} = bitcast<{stt}>({word(sub)});")
            if fn == "save":
                w("            return;")
            else:
                w(f"            return {tid_expr};")
            w("        }")
        w("        default: " + ("return;" if fn == "save" else "return 0xffffffffu;"))
        w("        }")
        w("    }")
        w("")
    # ---- bulk-copy restore: a tile's 32 entries of every slot column are 32
    # consecutive slots, so one cp.async.bulk per slot column brings the
    # tile into shared memory, where each lane reads its own entries
    stage_rows = []
    for qi in range(nq):
        stage_rows.append(sum(wdt for _, wdt, _ in layout[qi]["slots"]))
    max_stage = max(stage_rows) if stage_rows else 16
    max_stage = (max_stage + 15) // 16 * 16
    w("    // bytes of one queue entry's slots, the largest over the queues")
    w(f"    static constexpr unsigned kMaxStageRow = {max_stage}u;")
    w("    // Lane 0 of a warp: copies the full tile [toff, toff + 32) of queue q")
    w("    // (state half `base`) into `stage` (32 x kMaxStageRow bytes of shared")
    w("    // memory) with one bulk copy per slot column, completing on the")
    w("    // mbarrier at `mbar`; false (nothing issued) when an address is not on")
    w("    // a 16-byte boundary.")
    w("    __device__ __forceinline__ static bool")
    w("    bulk_issue(const int q, unsigned char* stage, const char* base, const unsigned cap, const unsigned toff,")
    w("               unsigned long long* mbar)")
    w("    {")
    w("        unsigned bytes = 0;")
    w("        switch(q)")
    w("        {")
    for qi in range(nq):
        w(f"        case {qi}: bytes = {32 * stage_rows[qi]}u; break;")
    w("        default: return false;")
    w("        }")
    w("        if((reinterpret_cast<unsigned long long>(base) | reinterpret_cast<unsigned long long>(stage)) & 15ull) return false;")
    w("        bulk_expect(mbar, bytes);")
    w("        switch(q)")
    w("        {")
    for qi in range(nq):
        w(f"        case {qi}:")
        so = 0
        for off, wdt, _ in layout[qi]["slots"]:
            w(f"            bulk_copy(stage + {so}u, base + {off}ull * cap + static_cast<unsigned long long>(toff) * {wdt}u, {32 * wdt}u, mbar);")
            so += 32 * wdt
        w("            break;")
    w("        default: break;")
    w("        }")
    w("        return true;")
    w("    }")
    w("")
    w("    // A lane's entry of a tile staged by bulk_issue; returns its thread id.")
    w("    __device__ __forceinline__ static unsigned")
    w("    restore_stage(const int q, Regs& R, const unsigned char* stage, const unsigned lane)")
    w("    {")
    w("        switch(q)")
    w("        {")
    for qi, (b, kk) in enumerate(queues):
        w(f"        case {qi}:")
        w("        {")
        if kk is not None:
            v = disp[b][0]
            w(f"            R.r{v} = static_cast<{CTYPE[L.regs[v].storage]}>({kk});")
        tid_expr = None
        so = 0
        for si, (off, wdt, contents) in enumerate(layout[qi]["slots"]):
            vt = {16: "uint4", 8: "uint2", 4: "unsigned", 2: "unsigned short", 1: "unsigned char"}[wdt]
            slot = f"reinterpret_cast<const {vt}*>(stage + {so}u)[lane]"
            so += 32 * wdt
            if wdt <= 2:
                (r, _), = contents
                w(f"            R.r{r} = bitcast<{CTYPE[L.regs[r].storage]}>({slot});")
                continue
            words = ["x", "y", "z", "w"][: wdt // 4] if wdt > 4 else [None]

            def word(sub, si=si, words=words):
                return f"v{si}" if words == [None] else f"v{si}.{words[sub // 4]}"

            w(f"            const {vt} v{si} = {slot};")
            for it, sub in contents:
                if it == "tid":
                    tid_expr = word(sub)
                elif L.regs[it].nbytes == 8:
                    w(f"            R.r{it} = bitcast<{CTYPE[L.regs[it].storage]}>((static_cast<unsigned long long>({word(sub + 4)}) << 32) | {word(sub)});")
                else:
                    w(f"            R.r{it} = bitcast<{CTYPE[L.regs[it].storage]}>({word(sub)});")
        w(f"            return {tid_expr};")
        w("        }")
    w("        default: return 0xffffffffu;")
    w("        }")
    w("    }")
    w("};")
    w("")
    # ---- host side
    w("const int kInTypes[] = {" + ", ".join(ABI_TYPE[t] for _, t, _ in k.inputs) + "};")
    w("const int kOutTypes[] = {" + ", ".join(ABI_TYPE[t] for _, t, _ in k.outputs) + "};")
    w("const char* const kInNames[] = {" + ", ".join(f'"{n}"' for _, _, n in k.inputs) + "};")
    w("const char* const kOutNames[] = {" + ", ".join(f'"{n}"' for _, _, n in k.outputs) + "};")
    w(f"const uint32_t kInstrs[] = {{{', '.join(map(str, counts))}}};")
    w(f"const uint32_t kLive[] = {{{', '.join(map(str, live_bytes))}}};")
    state_size = sum(r.nbytes for r in k.regs)
    w("")
    w("const loom_b200_kernel_info kInfo = {")
    w(f'    "{name}", "{k.digest()}", {nin}u, {nout}u, kInTypes, kOutTypes, kInNames, kOutNames,')
    w(f"    {nb}u, {len(k.regs)}u, {state_size}u, {len(state)}u, kInstrs, kLive}};")
    w("")
    # queue layouts for state inspection: the block (and dispatch context)
    # of each queue, its columns in save order and where they lie in a row
    assert all(rg.idx == i for i, rg in enumerate(k.regs)), "registers out of order"
    assert all(qk is None or -(2**31) <= qk < 2**31 for _, qk in queues), "dispatch context out of range"
    for qi, (qb, qk) in enumerate(queues):
        # columns in register-size order (the order of the queue analysis)
        cols = sorted(layout[qi]["cols"], key=lambda r: (-L.regs[r].nbytes, r))
        layout[qi]["order"] = cols
        if cols:
            at = layout[qi]["cols"]
            w(f"const uint32_t kQRegs{qi}[] = {{{', '.join(f'{r}u' for r in cols)}}};")
            w(f"const int kQTypes{qi}[] = {{{', '.join(ABI_TYPE[L.regs[r].storage] for r in cols)}}};")
            names = ", ".join('"' + k.regs[r].name + '"' for r in cols)
            w(f"const char* const kQNames{qi}[] = {{{names}}};")
            w(f"const unsigned long long kQOffs{qi}[] = {{{', '.join(f'{at[r][0]}ull' for r in cols)}}};")
            w(f"const unsigned kQSubs{qi}[] = {{{', '.join(f'{at[r][1]}u' for r in cols)}}};")
            w(f"const unsigned kQWidths{qi}[] = {{{', '.join(f'{at[r][2]}u' for r in cols)}}};")
    w("const loom_b200_queue_layout kQueues[] = {")
    for qi, (qb, qk) in enumerate(queues):
        cols = layout[qi]["order"]
        if cols:
            w(f"    {{{qb}u, {-1 if qk is None else qk}, {len(cols)}u, kQRegs{qi}, kQTypes{qi}, kQNames{qi}}},")
        else:
            w(f"    {{{qb}u, {-1 if qk is None else qk}, 0u, nullptr, nullptr, nullptr}},")
    w("};")
    w("const QueueSegment kSegments[] = {")
    for qi in range(nq):
        has = bool(layout[qi]["order"])
        offs = f"kQOffs{qi}, kQSubs{qi}, kQWidths{qi}" if has else "nullptr, nullptr, nullptr"
        t = layout[qi]["tid"]
        w(f"    {{{offs}, {t[0]}ull, {t[1]}u, {t[2]}u}},")
    w("};")
    w("")
    w("cudaError_t launch_plain(const PlainLaunch& a)")
    w("{")
    w("    const unsigned long long grid = (a.n + a.block - 1) / a.block;")
    w("    if(grid == 0) return cudaSuccess;")
    w("    if(a.profile)")
    w("        plain_kernel<K, true><<<static_cast<unsigned>(grid), a.block, 0, a.stream>>>(")
    w("            a.cols, a.first, a.n, a.max_steps, a.status, a.counters);")
    w("    else")
    w("        plain_kernel<K, false><<<static_cast<unsigned>(grid), a.block, 0, a.stream>>>(")
    w("            a.cols, a.first, a.n, a.max_steps, a.status, a.counters);")
    w("    return cudaGetLastError();")
    w("}")
    w("")
    caps = reg_caps(k)
    w(f"const unsigned kRegCaps[] = {{{', '.join(f'{c}u' for c in caps)}}};")
    w("")
    w("/// The megakernel at register cap `regs` (0: the default), in its form")
    w("/// for launches that never park when `park` is false; profiled launches")
    w("/// and launches with the staged restore (`bulk`) use the default cap and")
    w("/// the parking form.  NULL: no such cap compiled.")
    w("const void* regroup_fn(unsigned regs, bool profile, bool bulk, bool park)")
    w("{")
    w("    if(profile) return reinterpret_cast<const void*>(&regroup_kernel<K, true, K::kRegroupMaxRegs, true>);")
    w("    if(bulk) return reinterpret_cast<const void*>(&regroup_kernel<K, false, K::kRegroupMaxRegs, true>);")
    w("    switch(regs)")
    w("    {")
    w("    case 0u:")
    for c in caps:
        w(f"    case {c}u: return park ? reinterpret_cast<const void*>(&regroup_kernel<K, false, {c}, false, true>)")
        w(f"                          : reinterpret_cast<const void*>(&regroup_kernel<K, false, {c}, false, false>);")
    w("    default: return nullptr;")
    w("    }")
    w("}")
    w("")
    w("cudaError_t launch_regroup(const RegroupLaunch& a)")
    w("{")
    w("    void* args[] = {const_cast<RegroupParams*>(&a.params)};")
    w("    const void* fn = regroup_fn(a.regs, a.profile, a.params.bulk_restore != 0u, a.park);")
    w("    if(!fn) return cudaErrorInvalidValue;")
    w("    if(a.dyn_smem)")
    w("    {")
    w("        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,")
    w("                                                   static_cast<int>(a.dyn_smem));")
    w("        if(e != cudaSuccess) return e;")
    w("    }")
    w("    if(a.ordinary && a.params.slice_rounds == 1u)")
    w("        return cudaLaunchKernel(fn, dim3(a.grid), dim3(a.block), args, a.dyn_smem, a.stream);")
    w("    return cudaLaunchCooperativeKernel(fn, dim3(a.grid), dim3(a.block), args, a.dyn_smem, a.stream);")
    w("}")
    w("")
    w("cudaError_t regroup_occupancy(int block, bool profile, unsigned regs, unsigned dyn_smem, bool park, int* ctas)")
    w("{")
    w("    const void* fn = regroup_fn(regs, profile, dyn_smem != 0u, park);")
    w("    if(!fn) return cudaErrorInvalidValue;")
    w("    if(dyn_smem)")
    w("    {")
    w("        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,")
    w("                                                   static_cast<int>(dyn_smem));")
    w("        if(e != cudaSuccess) return e;")
    w("    }")
    w("    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, dyn_smem);")
    w("}")
    w("")
    w(f"}} }} // namespace loom_b200::k_{name}")
    w("")
    w(f"extern const loom_b200::KernelEntry loom_b200_entry_{name};")
    w(f"const loom_b200::KernelEntry loom_b200_entry_{name} = {{")
    w(f"    &loom_b200::k_{name}::kInfo, loom_b200::k_{name}::K::kRowBytes, {nq},")
    w(f"    &loom_b200::k_{name}::launch_plain, &loom_b200::k_{name}::launch_regroup,")
    w(f"    &loom_b200::k_{name}::regroup_occupancy,")
    w(f"    loom_b200::k_{name}::kQueues, loom_b200::k_{name}::kSegments,")
    w(f"    loom_b200::k_{name}::kRegCaps, {len(caps)}u, loom_b200::k_{name}::K::kMaxStageRow}};")
    return "\n".join(o) + "\n"


def generate_registry(names: List[str]) -> str:
    o = ["// Generated by loom_b200.codegen: the kernels compiled into libloom_b200.", ""]
    o.append('#include "../runtime_iface.h"')
    o.append("")
    for n in names:
        o.append(f"extern const loom_b200::KernelEntry loom_b200_entry_{n};")
    o.append("")
    o.append("namespace loom_b200 {")
    o.append("const KernelEntry* const kRegistry[] = {")
    for n in names:
        o.append(f"    &loom_b200_entry_{n},")
    o.append("};")
    o.append(f"const int kRegistrySize = {len(names)};")
    o.append("} // namespace loom_b200")
    return "\n".join(o) + "\n"
