"""The CPU gang port (Loom's compact and hybrid methods restated for g++,
oracle/gang_engine.hpp + oracle/gang_emit.py) against Loom's scalar backend.

The port is the multi-core CPU baseline of the hybrid method beside bse; it
computes every instruction as Loom's own semantics define it, so its
outputs must equal the golden fixtures (vm::bse::function<K>) bit for bit in
both methods, with one worker or several, whatever the stream size.
"""

import numpy as np
import pytest

from loom_b200.codegen import ir
from oracle import build_gang
from oracle import oracle as O

KERNELS = ir.available()

# Loom's own path tracers sample up to 64 times per pixel: a seeded subset
SUBSET = {"pt_const_40": 48, "pt2_const_40": 48, "pt_const_512": 48, "pt2_const_512": 48,
          "primary_const_256": 160, "primary_const_b20_256": 160, "sphere_pt_f32": 512}


@pytest.fixture(scope="module", autouse=True)
def port():
    build_gang.build()


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def _case(name, golden, golden_extra):
    ins, outs = golden(name)
    if name in SUBSET:
        idx = np.sort(O.uniform_int(11, SUBSET[name], 0, len(ins[0]) - 1).astype(np.int64))
        ins = [a[idx] for a in ins]
        outs = [a[idx] for a in outs]
    return ins, outs, golden_extra(name).get("table")


@pytest.mark.parametrize("method", ["compact", "hybrid"])
@pytest.mark.parametrize("name", KERNELS)
def test_port_matches_bse(name, method, golden, golden_extra):
    ins, outs, table = _case(name, golden, golden_extra)
    got = O.gang_run(name, ins, len(outs[0]), threads=1, table=table, method=method)
    for g, o in zip(got, outs):
        assert np.array_equal(_bits(g), _bits(o)), (name, method)


@pytest.mark.parametrize("name", ["fib_u64", "collatz_u64", "fac_u32", "jmp4_u64", "sphere_pt_f32", "union_cmov_f32"])
@pytest.mark.parametrize("threads,stream,utr", [(4, 64, 16), (3, 8, 2), (2, 1024, 8)])
def test_port_workers_and_streams(name, threads, stream, utr, golden, golden_extra):
    """Several workers drawing from one cursor, streams smaller and larger
    than the input, other thresholds: the same outputs."""
    ins, outs, table = _case(name, golden, golden_extra)
    st = {}
    got = O.gang_run(name, ins, len(outs[0]), threads=threads, table=table, stream=stream, utr_den=utr, stats=st)
    for g, o in zip(got, outs):
        assert np.array_equal(_bits(g), _bits(o)), name
    assert st["blocks"] > 0 and 0 < st["lanes"] <= st["blocks"] * 64


@pytest.mark.parametrize("n", [0, 1, 7, 17])
@pytest.mark.parametrize("method", ["compact", "hybrid"])
def test_port_ragged_sizes(n, method, golden):
    """Fewer threads than a gang, a gang and a bit, none at all."""
    (a,), (want,) = golden("fib_u64")
    got = O.gang_run("fib_u64", [a[:n]], n, threads=2, method=method)
    assert np.array_equal(got[0], want[:n])


def test_port_null_input_is_thread_index():
    """A NULL input column is the thread index, as in the bse runner."""
    n = 300
    got = O.gang_run("fib_u64", [None], n, method="hybrid")
    want = O.val_fib(np.arange(n, dtype=np.uint64))
    assert np.array_equal(got[0], want)


def test_port_hybrid_regroups():
    """The hybrid method runs fuller gangs than compact on a divergent kernel
    (the point of regrouping: Loom src/vm/simd.hpp:4105-4180)."""
    n = 4096
    a = O.uniform_int(5, n, 1, (1 << 32) - 1).astype(np.uint64)
    eff = {}
    for method in ("compact", "hybrid"):
        st = {}
        O.gang_run("collatz_u64", [a], n, method=method, stats=st)
        eff[method] = st["lanes"] / (st["blocks"] * 8)
    assert eff["hybrid"] > eff["compact"]
