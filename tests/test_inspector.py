"""State inspection without a GPU: the queue layouts the library reports
agree with the code generator's own queue analysis of every kernel's IR,
and the inspector's table prints parked rows as Loom's print_state prints a
thread (src/vm/dbg.hpp:918-933: PC label, then registers)."""

import numpy as np
import pytest

from loom_b200 import api
from loom_b200 import inspector as I
from loom_b200.codegen import ir


@pytest.mark.parametrize("name", ir.available())
def test_queue_layout_matches_the_ir(name):
    k = ir.load(name)
    want = k.queues()
    live = k.queue_liveness()
    got = api.queues(name)
    assert len(got) == len(want)
    for q, (b, ctx), lv in zip(got, want, live):
        assert q["block"] == b
        assert q["context"] == (-1 if ctx is None else ctx)
        assert sorted(r for r, _, _ in q["cols"]) == sorted(lv)
        for r, nm, t in q["cols"]:
            assert nm == k.regs[r].name
            assert t == k.regs[r].storage


def test_collatz_queues():
    qs = api.queues("collatz_u64")
    assert [(q["block"], q["context"]) for q in qs] == [(0, -1), (1, -1)]
    assert [c[1] for c in qs[0]["cols"]] == ["n"]
    assert sorted(c[1] for c in qs[1]["cols"]) == ["n", "steps"]


def test_unknown_kernel_queues():
    with pytest.raises(api.LoomError):
        api.queues("no_such_kernel")


def test_format_parked_prints_label_and_registers():
    parked = [
        dict(queue=1, block=1, context=-1, rows=3, tid=np.array([5, 9, 11], np.uint32),
             regs={"n": np.array([16, 8, 4], np.uint64), "steps": np.array([3, 2, 1], np.uint32)}),
        dict(queue=4, block=0, context=-1, rows=1, tid=np.array([2], np.uint32),
             regs={"x": np.array([0.5], np.float32)}),
        dict(queue=7, block=9, context=3, rows=2, tid=np.array([1, 4], np.uint32), regs={}),
    ]
    text = I.format_parked(parked, rows=2)
    lines = text.splitlines()
    assert lines[0] == "6 parked threads in 3 queues"
    assert "B1: 3 threads" in lines
    assert "START: 1 threads" in lines
    assert "B9<3>: 2 threads" in lines
    row = lines[lines.index("B1: 3 threads") + 2].split()
    assert row == ["5", "16", "3"]
    # at most `rows` rows per queue
    assert lines[lines.index("B1: 3 threads") + 4] == ""


def test_inspector_inputs_follow_the_kernel_types():
    cols = I._inputs("collatz_u64", 1000, 1, 1 << 20, 3)
    assert len(cols) == 1 and cols[0].dtype == np.uint64
    assert cols[0].min() >= 1 and cols[0].max() < (1 << 20)
    cols = I._inputs("union_f32", 10, 1, 100, 3)
    assert all(c.dtype == np.dtype(api.NP_TYPE[t]) for c, (_, t) in zip(cols, api.info("union_f32").inputs))
