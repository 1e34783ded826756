"""Parser and analyses for the text IR ("loomir") of a Loom kernel.

The IR is written by ``loom_b200/frontend/ir_emit.hpp`` from the kernel type
that Loom's own front end builds (``loom::vm::kernel_blank``, Loom
src/vm/core.hpp:939-1031).  A kernel is a list of basic blocks; block 0 is the
START block, target -1 is HALT (``halt_pos = index_t(-1)``, core.hpp:985).

Analyses provided here:

* successors per block (core.hpp:422-441);
* register liveness at block entry: the registers a parked thread must carry
  when it waits at a block.  Loom's hybrid backend stores every register of a
  row (src/vm/bve.hpp:494-693); the B200 regrouping engine stores only the
  live-in set of the block the thread waits at, which is what bounds its state
  traffic;
* static instruction counts per block (Compute + Jump + ParmJump), the unit of
  the VM-thread-instruction metric.
"""

from __future__ import annotations

import dataclasses
import hashlib
import pathlib
import struct
from typing import Dict, List, Optional, Sequence, Set, Tuple

HALT = -1

TYPE_BYTES = {
    "b8": 1,
    "i8": 1,
    "u8": 1,
    "i16": 2,
    "u16": 2,
    "i32": 4,
    "u32": 4,
    "i64": 8,
    "u64": 8,
    "f32": 4,
    "f64": 8,
}

INT_TYPES = {"b8", "i8", "u8", "i16", "u16", "i32", "u32", "i64", "u64"}
FLOAT_TYPES = {"f32", "f64"}


@dataclasses.dataclass(frozen=True)
class Operand:
    """A typed register view (``reg`` set) or a literal (``bits`` set)."""

    type: str
    reg: Optional[int] = None
    bits: Optional[int] = None

    @property
    def is_literal(self) -> bool:
        return self.reg is None

    def value(self):
        """Python value of a literal (int for integer types, float for fp)."""
        assert self.bits is not None
        t = self.type
        if t == "f32":
            return struct.unpack("<f", struct.pack("<I", self.bits))[0]
        if t == "f64":
            return struct.unpack("<d", struct.pack("<Q", self.bits))[0]
        nbits = TYPE_BYTES[t] * 8
        v = self.bits & ((1 << nbits) - 1)
        if t.startswith("i") and v >= 1 << (nbits - 1):
            v -= 1 << nbits
        return v

    def __str__(self) -> str:
        if self.is_literal:
            return f"k{self.type}:{self.bits:#x}"
        return f"r{self.reg}:{self.type}"


@dataclasses.dataclass
class Compute:
    op: str
    optype: Tuple[str, ...]  # functor operand type(s); () for generic ops
    dst: Operand
    args: List[Operand]
    consts: List[Operand]

    def reads(self) -> List[int]:
        return [a.reg for a in self.args if not a.is_literal]

    def writes(self) -> List[int]:
        return [self.dst.reg]


@dataclasses.dataclass
class Jump:
    target: int

    def reads(self) -> List[int]:
        return []

    def writes(self) -> List[int]:
        return []


@dataclasses.dataclass
class ParmJump:
    var: Operand
    targets: List[int]

    def reads(self) -> List[int]:
        return [] if self.var.is_literal else [self.var.reg]

    def writes(self) -> List[int]:
        return []


@dataclasses.dataclass
class Register:
    idx: int
    name: str
    nbytes: int
    types: List[str]

    @property
    def is_union(self) -> bool:
        return len(self.types) > 1

    @property
    def storage(self) -> str:
        """Storage type of the register in device code."""
        if not self.is_union:
            return self.types[0]
        return {1: "u8", 2: "u16", 4: "u32", 8: "u64"}[self.nbytes]


@dataclasses.dataclass
class Block:
    idx: int
    label: str
    instrs: list

    @property
    def terminator(self):
        if self.instrs and isinstance(self.instrs[-1], (Jump, ParmJump)):
            return self.instrs[-1]
        return None

    def successors(self) -> List[int]:
        t = self.terminator
        if t is None:
            return [HALT]
        if isinstance(t, Jump):
            return [t.target]
        return list(t.targets)


@dataclasses.dataclass
class Kernel:
    name: str
    index_type: str
    straight: bool
    regs: List[Register]
    inputs: List[Tuple[int, str, str]]  # (reg, type, name)
    outputs: List[Tuple[int, str, str]]
    blocks: List[Block]
    text: str

    # ------------------------------------------------------------ queries
    @property
    def num_blocks(self) -> int:
        return len(self.blocks)

    def pc_reg(self) -> Optional[int]:
        for r in self.regs:
            if r.name == "PC":
                return r.idx
        return None

    def digest(self) -> str:
        return structural_digest(self.text)

    def instr_counts(self) -> List[int]:
        return [len(b.instrs) for b in self.blocks]

    def succ_table(self) -> List[List[int]]:
        return [b.successors() for b in self.blocks]

    # ------------------------------------------------------------ liveness
    def liveness(self) -> Tuple[List[Set[int]], List[Set[int]]]:
        """Live-in and live-out register sets of every block.

        HALT behaves as a block that reads the output registers.  The PC
        register is never live: the engine keeps the PC outside the register
        file (it is the queue a thread waits in).
        """
        pc = self.pc_reg()
        use: List[Set[int]] = []
        defs: List[Set[int]] = []
        for b in self.blocks:
            u: Set[int] = set()
            d: Set[int] = set()
            for ins in b.instrs:
                for r in ins.reads():
                    if r not in d:
                        u.add(r)
                for r in ins.writes():
                    d.add(r)
            u.discard(pc)
            d.discard(pc)
            use.append(u)
            defs.append(d)
        halt_use = {r for r, _, _ in self.outputs}
        live_in = [set() for _ in self.blocks]
        live_out = [set() for _ in self.blocks]
        changed = True
        while changed:
            changed = False
            for i in reversed(range(self.num_blocks)):
                out: Set[int] = set()
                for s in self.blocks[i].successors():
                    out |= halt_use if s == HALT else live_in[s]
                new_in = use[i] | (out - defs[i])
                if out != live_out[i] or new_in != live_in[i]:
                    live_out[i] = out
                    live_in[i] = new_in
                    changed = True
        return live_in, live_out

    # ------------------------------------------------------------ dispatch
    def predecessors(self) -> List[List[int]]:
        preds: List[List[int]] = [[] for _ in self.blocks]
        for b in self.blocks:
            for t in b.successors():
                if t != HALT and b.idx not in preds[t]:
                    preds[t].append(b.idx)
        return preds

    def dispatch_blocks(self) -> Dict[int, Tuple[int, Dict[int, int]]]:
        """Blocks used as subroutines: block D ends with a ParmJump on a
        register v that D does not write, and every predecessor of D last
        writes v with a literal k before reaching D (Loom kernels call shared
        code this way, e.g. the RNG block of src/smallpt/vm/pt.hpp:889-914).
        Returns {D: (v, {k: target})}; the target of each context is known
        statically, which makes liveness context sensitive."""
        out: Dict[int, Tuple[int, Dict[int, int]]] = {}
        preds = self.predecessors()
        for b in self.blocks:
            t = b.terminator
            if not isinstance(t, ParmJump) or t.var.is_literal or b.idx == 0:
                continue
            v = t.var.reg
            if any(v in ins.writes() for ins in b.instrs):
                continue
            ctx: Dict[int, int] = {}
            ok = bool(preds[b.idx])
            for p in preds[b.idx]:
                last = None
                for ins in self.blocks[p].instrs:
                    if v in ins.writes():
                        last = ins
                if not (
                    isinstance(last, Compute)
                    and last.op == "mov"
                    and last.args[0].is_literal
                    and last.dst.reg == v
                ):
                    ok = False
                    break
                k = int(last.args[0].value())
                if not 0 <= k < len(t.targets) or self.blocks[p].successors() != [b.idx]:
                    ok = False
                    break
                ctx[k] = t.targets[k]
            if ok:
                out[b.idx] = (v, dict(sorted(ctx.items())))
        return out

    def queues(self) -> List[Tuple[int, Optional[int]]]:
        """Work queues of the regrouping engine: one per block (context k =
        None, the block's own live set) followed by one per context of every
        dispatch block."""
        q: List[Tuple[int, Optional[int]]] = [(b.idx, None) for b in self.blocks]
        for d, (_, ctx) in sorted(self.dispatch_blocks().items()):
            for k in ctx:
                q.append((d, k))
        return q

    def queue_liveness(self) -> List[Set[int]]:
        """Registers a thread parked in each queue must carry.

        Liveness runs on the CFG in which every dispatch block D is split
        into one copy per context k that jumps straight to its target, and
        each predecessor flows into the copy of the context it selects.  A
        queue (D, k) holds D's copy for context k without the dispatch
        register (restored as the constant k); queue (b, None) holds the live
        set of b on the split CFG (for D itself: the union over contexts)."""
        disp = self.dispatch_blocks()
        pc = self.pc_reg()
        nodes: List[Tuple[int, Optional[int]]] = self.queues()
        index = {n: i for i, n in enumerate(nodes)}
        use: List[Set[int]] = []
        defs: List[Set[int]] = []
        for b, _ in nodes:
            u: Set[int] = set()
            d: Set[int] = set()
            for ins in self.blocks[b].instrs:
                for r in ins.reads():
                    if r not in d:
                        u.add(r)
                for r in ins.writes():
                    d.add(r)
            u.discard(pc)
            d.discard(pc)
            use.append(u)
            defs.append(d)

        def succs(node) -> List[Tuple[int, Optional[int]]]:
            b, k = node
            if b in disp and k is not None:
                return [(disp[b][1][k], None)] if disp[b][1][k] != HALT else [(HALT, None)]
            out = []
            for t in self.blocks[b].successors():
                if t != HALT and t in disp and b != t:
                    v = disp[t][0]
                    last = None
                    for ins in self.blocks[b].instrs:
                        if v in ins.writes():
                            last = ins
                    k2 = int(last.args[0].value())
                    out.append((t, k2))
                else:
                    out.append((t, None))
            return out

        halt_use = {r for r, _, _ in self.outputs}
        live = [set() for _ in nodes]
        changed = True
        while changed:
            changed = False
            for i in reversed(range(len(nodes))):
                out: Set[int] = set()
                for s in succs(nodes[i]):
                    out |= halt_use if s[0] == HALT else live[index[s]]
                new = use[i] | (out - defs[i])
                if new != live[i]:
                    live[i] = new
                    changed = True
        # a context queue does not store its dispatch register
        for i, (b, k) in enumerate(nodes):
            if k is not None:
                live[i] = live[i] - {disp[b][0]}
        # the plain queue of a dispatch block: union over its contexts plus
        # the dispatch register (fallback for values outside the contexts)
        for d, (v, ctx) in disp.items():
            u: Set[int] = set()
            for k in ctx:
                u |= live[index[(d, k)]]
            live[index[(d, None)]] = u | {v}
        return live

    def rpo_ranks(self) -> List[int]:
        """Rank of every block in reverse post-order of a depth-first walk
        from START (loop headers before their bodies, a join after both of
        its branches); unreachable blocks come last."""
        seen = [False] * self.num_blocks
        post: List[int] = []
        stack = [(0, iter(self.blocks[0].successors()))] if self.blocks else []
        if self.blocks:
            seen[0] = True
        while stack:
            b, it = stack[-1]
            nxt = next((t for t in it if t != HALT and not seen[t]), None)
            if nxt is None:
                post.append(b)
                stack.pop()
            else:
                seen[nxt] = True
                stack.append((nxt, iter(self.blocks[nxt].successors())))
        order = list(reversed(post)) + [b for b in range(self.num_blocks) if not seen[b]]
        rank = [0] * self.num_blocks
        for r, b in enumerate(order):
            rank[b] = r
        return rank

    def state_regs(self) -> List[int]:
        """Registers that are live at the entry of some block: the columns of
        the regrouping engine's state file."""
        live_in, _ = self.liveness()
        s: Set[int] = set()
        for li in live_in:
            s |= li
        return sorted(s)


def structural_digest(text: str) -> str:
    """FNV-1a (64-bit) of the IR without its `kernel <name>` line, as 16 hex
    digits: two kernel types with the same program get the same digest
    whatever they are called (the C++ front end computes the same value)."""
    h = 0xCBF29CE484222325
    for ln in text.splitlines(keepends=True):
        if ln.startswith("kernel "):
            continue
        for byte in ln.encode():
            h ^= byte
            h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return f"{h:016x}"


# ---------------------------------------------------------------- parsing
def _operand(tok: str) -> Operand:
    if tok.startswith("r"):
        reg, t = tok[1:].split(":")
        return Operand(type=t, reg=int(reg))
    if tok.startswith("k"):
        t, bits = tok[1:].split(":")
        return Operand(type=t, bits=int(bits, 16))
    raise ValueError(f"bad operand {tok!r}")


def parse(text: str) -> Kernel:
    lines = [ln.strip() for ln in text.splitlines() if ln.strip()]
    if not lines or lines[0] != "loomir 1":
        raise ValueError("not a loomir 1 file")
    name = ""
    index_type = ""
    straight = False
    regs: List[Register] = []
    inputs: List[Tuple[int, str, str]] = []
    outputs: List[Tuple[int, str, str]] = []
    blocks: List[Block] = []
    cur: Optional[Block] = None
    for ln in lines[1:]:
        tok = ln.split()
        kind = tok[0]
        if kind == "kernel":
            name = tok[1]
        elif kind == "index":
            index_type = tok[1]
        elif kind == "straight":
            straight = tok[1] == "1"
        elif kind == "reg":
            regs.append(Register(int(tok[1]), tok[2], int(tok[3]), tok[4].split(",")))
        elif kind == "input":
            inputs.append((int(tok[1]), tok[2], tok[3]))
        elif kind == "output":
            outputs.append((int(tok[1]), tok[2], tok[3]))
        elif kind == "block":
            cur = Block(int(tok[1]), tok[2], [])
            blocks.append(cur)
        elif kind == "i":
            assert cur is not None
            rest = tok[3:]
            consts: List[Operand] = []
            if "|" in rest:
                cut = rest.index("|")
                consts = [_operand(t) for t in rest[cut + 1 :]]
                rest = rest[:cut]
            optype = () if tok[2] == "-" else tuple(tok[2].split(","))
            ops = [_operand(t) for t in rest]
            cur.instrs.append(Compute(tok[1], optype, ops[0], ops[1:], consts))
        elif kind == "j":
            assert cur is not None
            cur.instrs.append(Jump(int(tok[1])))
        elif kind == "p":
            assert cur is not None
            cur.instrs.append(ParmJump(_operand(tok[1]), [int(t) for t in tok[2:]]))
        elif kind == "end":
            break
        else:
            raise ValueError(f"bad IR line {ln!r}")
    k = Kernel(name, index_type, straight, regs, inputs, outputs, blocks, text)
    _validate(k)
    return k


def _validate(k: Kernel) -> None:
    nb = k.num_blocks
    if nb == 0:
        raise ValueError(f"{k.name}: no blocks")
    for b in k.blocks:
        for s in b.successors():
            if s != HALT and not 0 <= s < nb:
                raise ValueError(f"{k.name}: block {b.idx} jumps to {s}")
    for r in k.regs:
        for t in r.types:
            if TYPE_BYTES[t] != r.nbytes:
                raise ValueError(f"{k.name}: register {r.name} mixes sizes")


IR_DIR = pathlib.Path(__file__).resolve().parent.parent / "ir"


def load(name: str, ir_dir: Optional[pathlib.Path] = None) -> Kernel:
    d = ir_dir or IR_DIR
    return parse((d / f"{name}.lir").read_text())


def available(ir_dir: Optional[pathlib.Path] = None) -> List[str]:
    d = ir_dir or IR_DIR
    return sorted(p.stem for p in d.glob("*.lir"))
