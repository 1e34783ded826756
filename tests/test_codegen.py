"""The code generator's tables against independent restatements (CPU only):
block ranks in reverse post-order, loop headers, the regrouping cost
model's per-block quorum, and the register cap of the megakernel, for
every kernel of the registry."""

import math
import pathlib
import re

import pytest

from loom_b200.codegen import emit_cuda as E
from loom_b200.codegen import ir
from loom_b200.codegen.ir import HALT

GEN = pathlib.Path(__file__).resolve().parents[1] / "loom_b200" / "csrc" / "gen"
KERNELS = ir.available()


def _table(src: str, name: str):
    m = re.search(rf"__constant__ (?:unsigned|int) {name}\[\d+\] = \{{([^}}]*)\}};", src)
    assert m, name
    return [int(x) for x in m.group(1).split(",")]


@pytest.mark.parametrize("name", KERNELS)
def test_ranks_are_a_reverse_post_order(name):
    k = ir.load(name)
    rank = k.rpo_ranks()
    assert sorted(rank) == list(range(k.num_blocks))
    assert rank[0] == 0
    # reverse post-order of a depth-first walk: an edge that does not close a
    # cycle goes to a block of higher rank, so following only edges to
    # higher ranks never returns to a block, and every edge b -> t with
    # rank[t] <= rank[b] closes a cycle through t (t reaches b)
    succ = k.succ_table()

    def reaches(a, b):
        seen, todo = {a}, [a]
        while todo:
            x = todo.pop()
            if x == b:
                return True
            for t in succ[x]:
                if t != HALT and t not in seen:
                    seen.add(t)
                    todo.append(t)
        return False

    for b in range(k.num_blocks):
        if not reaches(0, b):
            continue  # unreachable blocks are ranked last, in index order
        for t in succ[b]:
            if t != HALT and rank[t] <= rank[b]:
                assert reaches(t, b), (name, b, t)


@pytest.mark.parametrize("name", KERNELS)
def test_generated_tables_match_the_ir(name):
    """kRankTab is the IR's reverse post-order; kQuorumTab is the cost
    model: a group of g lanes at block b runs it now (I_b warp instructions)
    or parks (C_b column stores, C_b loads per tile of 32, then I_b at full
    width), so parking pays while g < 32 (I_b - C_b) / (I_b + C_b), capped
    at 28; C_b = live registers of the block's widest queue + the thread id."""
    k = ir.load(name)
    src = (GEN / f"{name}.cu").read_text()
    assert _table(src, "kRankTab") == k.rpo_ranks()
    assert _table(src, "kInstrTab") == k.instr_counts()
    qlive = k.queue_liveness()
    want = []
    for b, ib in enumerate(k.instr_counts()):
        c = max((len(qlive[q]) for q, (qb, _) in enumerate(k.queues()) if qb == b), default=0) + 1
        want.append(min(28, max(0, math.ceil(32 * (ib - c) / (ib + c)))) if ib > c else 0)
    assert _table(src, "kQuorumTab") == want
    assert f"static constexpr int kRegroupMaxRegs = {E.REGROUP_MAX_REGS};" in src


def test_collatz_loop_header_and_quorum():
    k = ir.load("collatz_u64")
    rank = k.rpo_ranks()
    headers = {t for b in k.blocks for t in b.successors() if t != HALT and rank[t] <= rank[b.idx]}
    assert headers == {1}
    src = (GEN / "collatz_u64.cu").read_text()
    # START: 3 instructions, 1 live register (n) -> ceil(32 * 1 / 5) = 7;
    # loop: 8 instructions, 2 live registers (n, steps) -> ceil(32 * 5 / 11) = 15
    assert _table(src, "kQuorumTab") == [7, 15]


@pytest.mark.parametrize("name", KERNELS)
def test_queue_rows_pack_every_live_register_once(name):
    """The queue row layout (16-byte slots): every live register of every
    queue and the thread id sit in exactly one slot, at an offset inside the
    slot that is a multiple of their size, without overlapping; slots of 16,
    8 or 4 bytes hold only 4- and 8-byte values, narrow registers get slots
    of their own; the segments of the queues follow one another and every
    segment ends on 8 bytes."""
    k = ir.load(name)
    L = E.Lowering(k)
    qlive = k.queue_liveness()
    start = 0
    for q in range(len(k.queues())):
        lay = E.pack_slots([(r, L.regs[r].nbytes) for r in qlive[q]], start)
        seen = {}
        used = {}
        for off, width, contents in lay["slots"]:
            assert width in (1, 2, 4, 8, 16) and off >= start
            for it, sub in contents:
                n = 4 if it == "tid" else L.regs[it].nbytes
                assert it not in seen
                seen[it] = (off, sub, width)
                assert sub % n == 0 and sub + n <= width
                if width >= 4:
                    assert n in (4, 8)
                for byte in range(off + sub, off + sub + n):
                    assert byte not in used, (name, q, it)
                    used[byte] = it
        assert set(seen) == set(qlive[q]) | {"tid"}
        assert lay["cols"] == {r: seen[r] for r in qlive[q]} and lay["tid"] == seen["tid"]
        assert lay["end"] % 8 == 0 and lay["end"] >= max(used) + 1
        start = lay["end"]
    src = (GEN / f"{name}.cu").read_text()
    assert f"static constexpr unsigned long long kRowBytes = {start}ull;" in src


def test_slot_packing_of_a_mixed_row():
    """Two 8-byte and five 4-byte registers with the thread id: one slot of
    the two 8-byte values, one of four 4-byte values, one of the fifth and
    the id; a 1-byte register on its own."""
    lay = E.pack_slots([(0, 8), (1, 4), (2, 8), (3, 4), (4, 4), (5, 4), (6, 4), (7, 1)], 0)
    assert [(o, w, [i for i, _ in c]) for o, w, c in lay["slots"]] == [
        (0, 16, [0, 2]), (16, 16, [1, 3, 4, 5]), (32, 8, [6, "tid"]), (40, 1, [7])]
    assert lay["end"] == 48
