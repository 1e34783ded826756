"""Generator of the CPU gang port: C++ of one Loom kernel for N-lane gangs.

BASELINE INFRASTRUCTURE ONLY.  bench.py's CPU leg and tests/ use the port
built from this output (oracle/build_gang.py); the product never does.

Loom's compact and hybrid CPU backends (src/vm/simd.hpp:3739-4292) run a
gang of N threads (N = 64 bytes / the kernel's index type: 16 for a 32-bit
PC on AVX-512) through one basic block at a time: every instruction of the
block is computed for all N lanes as one vector operation and written back
only in the lanes whose PC is that block (compact_masked_block_compiler,
blend on every write).  Those backends need clang-only builtins and
range-v3, which are absent here, so this generator restates their block
execution from the kernel's text IR instead: each register becomes an
N-element array, each instruction a loop over the lanes whose result is
blended into the register under the block's lane mask (g++ turns the loops
into AVX-512 masked vector code), and the block's transfer writes the next
PC of its lanes.  The instruction semantics are those of the CUDA lowering
(loom_b200.codegen.emit_cuda.Lowering, Loom src/vm/operators.hpp), read
lane by lane; the host helpers they call (oracle/gang_engine.hpp) follow the
scalar backend bse (Loom src/vm/bse.hpp), so results equal bse's bit for
bit.  The gang driver (threaded dispatch, groups, counting sort, streams)
is the hand-written oracle/gang_engine.hpp.
"""

from __future__ import annotations

import pathlib
import sys
from typing import List

ROOT = pathlib.Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from loom_b200.codegen import ir  # noqa: E402
from loom_b200.codegen.emit_cuda import CTYPE, Lowering  # noqa: E402

# integer division and remainder trap on a zero divisor: computed only in
# the lanes that run the block (every other op, float division included, is
# computed in every lane and blended)
_TRAPPING = {"div", "mod"}

# kernels of at most this many instructions have their blocks inlined into
# the dispatch
_SMALL_KERNEL = 64

# libm calls stay scalar: made only for the lanes that run the block
_LIBM = {"sin", "cos"}

# a loop over the gang's lanes, kept as a loop (not unrolled) so that g++
# vectorises it whole
_LOOP = '_Pragma("GCC ivdep") _Pragma("GCC unroll 1") for(int l = 0; l < N; ++l)'


class LaneLowering(Lowering):
    """The CUDA lowering with every register read as lane `l` of its array."""

    def rname(self, idx: int) -> str:
        return f"R.r{idx}[l]"

    def value(self, dst: ir.Operand, expr: str) -> str:
        """`expr` converted to the destination view, as the register's
        storage type (the value `write` would store)."""
        reg = self.regs[dst.reg]
        val = f"static_cast<{CTYPE[dst.type]}>({expr})"
        if reg.storage == dst.type:
            return val
        return f"bitcast<{CTYPE[reg.storage]}>({val})"


def lanes_of(k: ir.Kernel) -> int:
    """Gang width: 64 bytes of the kernel's index type, as Loom's
    native_vector_extent_v<index_t> on AVX-512 (simd.hpp:3760)."""
    return max(1, 64 // ir.TYPE_BYTES[k.index_type])


def generate(k: ir.Kernel) -> str:
    L = LaneLowering(k)
    small = sum(k.instr_counts()) <= _SMALL_KERNEL
    name = k.name
    nb = k.num_blocks
    N = lanes_of(k)
    regs = [r for r in k.regs if r.idx != L.pc]
    succ = k.succ_table()
    o: List[str] = []
    w = o.append
    w(f"// Generated by oracle/gang_emit.py from loom_b200/ir/{name}.lir.")
    w("// CPU gang port of one Loom kernel (baseline infrastructure only).")
    w('#include "gang_engine.hpp"')
    w("")
    w(f"namespace loom_gang {{ namespace g_{name} {{")
    w("")
    w("struct G")
    w("{")
    w(f"    static constexpr int N = {N};")
    w(f"    static constexpr int kNumBlocks = {nb};")
    w(f"    static constexpr int kNumIn = {len(k.inputs)};")
    w(f"    static constexpr int kNumOut = {len(k.outputs)};")
    w("")
    # ---- gang registers and the stream's columns
    w("    struct Regs")
    w("    {")
    for r in regs:
        w(f"        alignas(64) {CTYPE[r.storage]} r{r.idx}[N]; // {r.name}")
    w("        alignas(64) int pc[N];")
    w("        alignas(64) unsigned long long tid[N];")
    w("    };")
    w("")
    w("    struct Mem")
    w("    {")
    for r in regs:
        w(f"        {CTYPE[r.storage]}* r{r.idx};")
    w("        int* pc;")
    w("        unsigned long long* tid;")
    w("    };")
    w("")
    w("    static size_t row_bytes()")
    w("    {")
    w(f"        return {sum(ir.TYPE_BYTES[r.storage] for r in regs)} + sizeof(int) + sizeof(unsigned long long);")
    w("    }")
    w("")
    w("    /// Columns of `rows` threads carved from `base` (64-byte aligned).")
    w("    static Mem carve(unsigned char* base, const size_t rows)")
    w("    {")
    w("        Mem m;")
    w("        size_t off = 0;")
    w("        auto take = [&](const size_t bytes) { unsigned char* p = base + off; off += (bytes + 63) / 64 * 64; return p; };")
    for r in regs:
        w(f"        m.r{r.idx} = reinterpret_cast<{CTYPE[r.storage]}*>(take(rows * sizeof({CTYPE[r.storage]})));")
    w("        m.pc = reinterpret_cast<int*>(take(rows * sizeof(int)));")
    w("        m.tid = reinterpret_cast<unsigned long long*>(take(rows * sizeof(unsigned long long)));")
    w("        return m;")
    w("    }")
    w("")
    w("    static size_t carve_bytes(const size_t rows)")
    w("    {")
    w("        size_t b = 0;")
    for r in regs:
        w(f"        b += (rows * sizeof({CTYPE[r.storage]}) + 63) / 64 * 64;")
    w("        b += (rows * sizeof(int) + 63) / 64 * 64 + (rows * sizeof(unsigned long long) + 63) / 64 * 64;")
    w("        return b;")
    w("    }")
    w("")
    w("    static void load(Regs& R, const Mem& m, const size_t pos)")
    w("    {")
    for r in regs:
        w(f"        std::memcpy(R.r{r.idx}, m.r{r.idx} + pos, sizeof R.r{r.idx});")
    w("        std::memcpy(R.pc, m.pc + pos, sizeof R.pc);")
    w("        std::memcpy(R.tid, m.tid + pos, sizeof R.tid);")
    w("    }")
    w("")
    w("    static void store(const Regs& R, const Mem& m, const size_t pos)")
    w("    {")
    for r in regs:
        w(f"        std::memcpy(m.r{r.idx} + pos, R.r{r.idx}, sizeof R.r{r.idx});")
    w("        std::memcpy(m.pc + pos, R.pc, sizeof R.pc);")
    w("        std::memcpy(m.tid + pos, R.tid, sizeof R.tid);")
    w("    }")
    w("")
    w("    /// Row `i` of `a` to row `j` of `b` (the counting sort's scatter).")
    w("    static void move(const Mem& a, const size_t i, const Mem& b, const size_t j)")
    w("    {")
    for r in regs:
        w(f"        b.r{r.idx}[j] = a.r{r.idx}[i];")
    w("        b.pc[j] = a.pc[i];")
    w("        b.tid[j] = a.tid[i];")
    w("    }")
    w("")
    # ---- thread start and finish
    w("    /// Loom's set_inputs: every register zero, then the inputs of thread")
    w("    /// `t` (a NULL column is the thread index), PC at START.")
    w("    static void start(const Mem& m, const size_t row, const void* const* in, const unsigned long long t)")
    w("    {")
    for r in regs:
        w(f"        m.r{r.idx}[row] = 0;")
    for i, (reg, t, vname) in enumerate(k.inputs):
        ct = CTYPE[t]
        src = f"(in[{i}] ? static_cast<const {ct}*>(in[{i}])[t] : static_cast<{ct}>(t))"
        rr = L.regs[reg]
        if rr.storage == t:
            w(f"        m.r{reg}[row] = {src}; // {vname}")
        else:
            w(f"        m.r{reg}[row] = bitcast<{CTYPE[rr.storage]}>({src}); // {vname}")
    w("        (void)in;")
    w(f"        m.pc[row] = {0 if nb else 'kNumBlocks'};")
    w("        m.tid[row] = t;")
    w("    }")
    w("")
    w("    static void finish(const Mem& m, const size_t row, void* const* out)")
    w("    {")
    w("        const unsigned long long t = m.tid[row];")
    for j, (reg, t, vname) in enumerate(k.outputs):
        ct = CTYPE[t]
        rr = L.regs[reg]
        val = f"m.r{reg}[row]" if rr.storage == t else f"bitcast<{ct}>(m.r{reg}[row])"
        w(f"        static_cast<{ct}*>(out[{j}])[t] = {val}; // {vname}")
    w("        (void)out; (void)t;")
    w("    }")
    w("")
    # ---- blocks
    for b, blk in enumerate(k.blocks):
        w(f"    // block {b}: {blk.label}")
        # the blocks of a large kernel stay functions of their own: inlined
        # into its dispatch, g++ compiled their lane loops worse (the path
        # tracers ran 3x slower); a small kernel's dispatch keeps them inline
        attr = "" if small else "__attribute__((noinline)) "
        w(f"    {attr}static void block_{b}(Regs& R, const Ctx& ctx)")
        w("    {")
        w("        (void)ctx;")
        # every lane loop selects by comparing the lane's PC with the block
        # (PCs change only in the block's last loop): one vector compare
        # per loop, at whatever width the destination has
        on = f"R.pc[l] == {b}"
        for ins in blk.instrs:
            if not isinstance(ins, ir.Compute):
                continue
            expr = L.value(ins.dst, L.expr(ins))
            d = f"R.r{ins.dst.reg}[l]"
            if ins.op in _LIBM or (ins.op in _TRAPPING and ins.optype and ins.optype[0] in ir.INT_TYPES):
                w(f"        {_LOOP} if({on}) {d} = {expr};")
            else:
                w(f"        {_LOOP} {{ const auto v = {expr}; {d} = ({on}) ? v : {d}; }}")
        nx = L.next_expr(blk).replace("kHalt", "kNumBlocks")
        w(f"        {_LOOP} {{ const int nx = {nx}; R.pc[l] = ({on}) ? nx : R.pc[l]; }}")
        w("    }")
        w("")
    # ---- threaded dispatch with the successors compiled in: each block's
    # successors in the order of its jump table, HALT as kNumBlocks (Loom
    # src/vm/core.hpp:418-441, the table threaded_dispatch::eval walks)
    w("    /// Loom's threaded dispatch (threaded_dispatch::eval) over this kernel:")
    w("    /// each block's exit counts the lanes at its successors (in jump-table")
    w("    /// order), adds those with lanes to the pending set and jumps to the")
    w("    /// fullest one while it holds more lanes than the threshold.")
    w("    static std::uint64_t run_from(int b, unsigned pops, Regs& R, std::uint64_t pending,")
    w("                                  const unsigned threshold, const Ctx& ctx, Counters& c)")
    w("    {")
    w("        switch(b)")
    w("        {")
    for b in range(nb):
        w(f"        case {b}: goto B{b};")
    w("        default: return pending;")
    w("        }")
    for b in range(nb):
        ss = succ[b]
        w(f"    B{b}:")
        w("        c.blocks += 1;")
        w("        c.lanes += pops;")
        w(f"        block_{b}(R, ctx);")
        w(f"        pending &= ~(1ull << {b});")
        if len(ss) == 1:
            t = ss[0]
            if t == ir.HALT:
                w("        return pending;")
            else:
                w(f"        {{ const unsigned p = pops_at<N>(R.pc, {t}); if(p > threshold) {{ pops = p; goto B{t}; }} }}")
                w("        return pending;")
        else:
            w("        {")
            w("            unsigned bp = 0;")
            w("            int bi = -1;")
            for i, t in enumerate(ss):
                tid = nb if t == ir.HALT else t
                keep = "" if t == ir.HALT else f" if(p) pending |= 1ull << {t};"
                w(f"            {{ const unsigned p = pops_at<N>(R.pc, {tid});{keep} if(p > bp) {{ bp = p; bi = {i}; }} }}")
            w("            if(bp > threshold)")
            w("            {")
            w("                pops = bp;")
            w("                switch(bi)")
            w("                {")
            for i, t in enumerate(ss):
                if t != ir.HALT:
                    w(f"                case {i}: goto B{t};")
            w("                default: break;")
            w("                }")
            w("            }")
            w("        }")
            w("        return pending;")
    w("    }")
    w("};")
    w("")
    w("}} // namespace")
    w("")
    w(f'extern "C" int loom_gang_run_{name}(const void* const* in, void* const* out, unsigned long long n,')
    w("                                   int threads, const unsigned* table, int method, unsigned stream,")
    w("                                   unsigned utr_den, unsigned long long* stats)")
    w("{")
    w(f"    return loom_gang::run<loom_gang::g_{name}::G>(in, out, n, threads, table, method, stream, utr_den, stats);")
    w("}")
    return "\n".join(o) + "\n"


def main(argv: List[str]) -> int:
    out = pathlib.Path(argv[1]) if len(argv) > 1 else ROOT / "oracle" / "_lib" / "gang"
    out.mkdir(parents=True, exist_ok=True)
    for name in ir.available():
        (out / f"{name}.cpp").write_text(generate(ir.load(name)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main(sys.argv))
