"""Parity of both B200 engines with Loom's scalar backend (needs a GPU).

Every kernel of the registry runs through the C ABI in plain and regrouping
form on the golden inputs and must reproduce Loom bse's outputs bit for bit
(tests/golden/, made by tests/golden/make_golden.py).  Large cases check
size-independent properties: plain == regroup on every thread, a seeded
sample against the C oracle, known answers, and the total VM-instruction
count equal to the oracle's (each executed block counted once per thread).
"""

import numpy as np
import pytest

from loom_b200 import api
from loom_b200.codegen import ir
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KERNELS = ir.available()


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def _as_list(x):
    return list(x) if isinstance(x, tuple) else [x]


# Bit-exact everywhere except where a kernel's float results go through the
# host libm's sinf/cosf, which the device matches to within an ulp (it
# evaluates them in double and rounds once): Loom's pt2_const_40 calls them
# on every bounce.  There every float output is held within ULP_TOLERANCE
# units in the last place of the scalar backend's value, and integer outputs
# (ray counts, pixel ids) stay exact.  A libm value one ulp apart is carried
# through the rest of the path's arithmetic: over all 262,144 pixels of the
# 512x512 render about 0.4 % differ, by at most 14 ulp.
ULP_TOLERANCE = {"pt2_const_40": 16, "pt2_const_512": 16}
# ... and the image those float outputs form (one radiance channel per
# output, one pixel per thread) within this relative RMSE:
# sqrt(mean((got - want)^2)) / sqrt(mean(want^2)).
IMAGE_RMSE_TOLERANCE = 1e-6


def image_rmse(got, want) -> float:
    g = np.asarray(got, dtype=np.float64)
    w = np.asarray(want, dtype=np.float64)
    ref = float(np.sqrt(np.mean(w * w))) if w.size else 0.0
    return float(np.sqrt(np.mean((g - w) ** 2))) / ref if ref > 0 else 0.0


def _check(name, got, want):
    for g, w in zip(got, want):
        if name in ULP_TOLERANCE and np.asarray(w).dtype.kind == "f":
            g, w = np.asarray(g), np.asarray(w)
            ulps = np.abs(g.astype(np.float64) - w.astype(np.float64)) / np.spacing(np.abs(w)).astype(np.float64)
            assert float(ulps.max()) <= ULP_TOLERANCE[name], f"{name}: {float(ulps.max())} ulp apart"
            assert image_rmse(g, w) <= IMAGE_RMSE_TOLERANCE, f"{name}: image RMSE {image_rmse(g, w):.3g}"
            continue
        assert np.array_equal(_bits(g), _bits(w)), f"{name}: {int((g != w).sum())} threads differ"


@pytest.mark.parametrize("mode", ["plain", "regroup"])
@pytest.mark.parametrize("name", KERNELS)
def test_engine_matches_loom_bse(name, mode, golden, golden_extra):
    ins, outs = golden(name)
    extra = golden_extra(name)
    n = len(ins[0])
    with api.Function(name, n, mode) as f:
        if "table" in extra:
            got = _as_list(f.launch_host(ins, n, table=extra["table"]))
        else:
            got = _as_list(f(*ins))
        s = f.stats(raise_on_device_error=True)
    _check(name, got, outs)
    assert s["threads"] == n


@pytest.mark.parametrize("mode", ["plain", "regroup"])
def test_path_tracer_instance_forms(mode, golden, golden_extra):
    """The batched path-tracing fixture (a Cornell render and three random
    scenes in one launch) with (instance, sample) computed on the device
    from the instance offsets instead of input arrays."""
    name = "sphere_pt_f32"
    ins, outs = golden(name)
    extra = golden_extra(name)
    n = len(ins[0])
    with api.Function(name, n, mode) as f:
        got = _as_list(
            f.launch_host(
                [api.Instance(), api.LocalIota()],
                n,
                instance_starts=extra["starts"],
                table=extra["table"],
            )
        )
        f.stats(raise_on_device_error=True)
    _check(name, got, outs)


def test_broadcast_input_form(golden):
    ins, outs = golden("collatz_u64")
    with api.Function("collatz_u64", 64, "regroup") as f:
        got = f.launch_host([api.Broadcast(27, "u64")], 64)
    assert (got == 111).all()


REGROUP_VARIANTS = [
    dict(utr_lanes=1, period=1),
    dict(utr_lanes=32, period=3),
    dict(utr_lanes=16, period=7, block_size=64),
    dict(utr_lanes=8, period=1000, block_size=1024),
    dict(population=100),
    dict(population=1000, utr_lanes=24),
    dict(prefetch=False, period=5),
    dict(burst=1, refill=False, spread_lanes=33),
    dict(burst=64, spread_lanes=1, utr_lanes=1),
    dict(ctas_per_sm=1, population=37),
    dict(burst=1, utr_lanes=4, population=64),
    dict(cost_model=True),
    dict(cost_model=True, burst=16, utr_lanes=24, population=512),
    dict(cost_model=True, burst=1, utr_lanes=1, period=2),
    dict(schedule=1),
    dict(schedule=1, utr_lanes=1, spread_lanes=1, burst=64),
    dict(schedule=1, cost_model=True, burst=8, population=300),
    dict(schedule=2, burst=16),
    dict(schedule=2, burst=3, period=7, population=100),
    # no period limit: schedule 2 never parks, one round, no queue state
    dict(schedule=2, burst=2, period=api.PERIOD_UNBOUNDED, prefetch=False),
    dict(schedule=2, burst=1, period=api.PERIOD_UNBOUNDED, prefetch=True, block_size=64),
    # whole warps of threads run plain-fashion inside the persistent kernel
    dict(schedule=3, burst=1 << 20, period=api.PERIOD_UNBOUNDED),
    dict(schedule=3, burst=1 << 20, period=api.PERIOD_UNBOUNDED, prefetch=False, population=100),
    dict(schedule=3, burst=2, period=9, population=300),
    # launches below plain_below threads run the plain engine
    dict(plain_below=1 << 40),
    # schedule 2 holding long blocks back until 8 or all lanes stand there
    dict(schedule=2, burst=2, period=api.PERIOD_UNBOUNDED, defer_lanes=8),
    dict(schedule=2, burst=4, period=api.PERIOD_UNBOUNDED, defer_lanes=32, prefetch=True),
    dict(schedule=2, burst=1, period=5, population=200, defer_lanes=12),
    # few self-loop iterations per step
    dict(schedule=2, burst=4, period=api.PERIOD_UNBOUNDED, spin_iters=3),
    # bursts that end once lanes have halted
    dict(schedule=2, burst=64, period=api.PERIOD_UNBOUNDED, refill_lanes=1),
    dict(schedule=2, burst=16, period=7, population=300, refill_lanes=4),
    # the never-park instantiation at another register cap, and a never-park
    # launch that asks for the staged restore (which then runs the parking form)
    dict(schedule=2, burst=2, period=api.PERIOD_UNBOUNDED, max_regs=48),
    dict(schedule=3, burst=1 << 20, period=api.PERIOD_UNBOUNDED, max_regs=40, block_size=128),
    dict(schedule=2, burst=2, period=api.PERIOD_UNBOUNDED, bulk_restore=True),
    # full tiles restored through shared memory with bulk copies
    dict(bulk_restore=True, utr_lanes=24, period=3, population=256),
    dict(bulk_restore=True, cost_model=True, burst=8, population=512, block_size=512),
]


@pytest.mark.parametrize("variant", REGROUP_VARIANTS, ids=lambda v: ",".join(f"{k}={x}" for k, x in v.items()))
@pytest.mark.parametrize(
    "name", ["fib_u64", "collatz_u64", "fac_u64", "jmp4_u64", "union_cmov_f32", "slt_inv_u32", "sphere_pt_f32", "pt_const_40"]
)
def test_regroup_options_keep_results(name, variant, golden, golden_extra):
    ins, outs = golden(name)
    extra = golden_extra(name)
    with api.Function(name, len(ins[0]), "regroup", **variant) as f:
        if "table" in extra:
            got = _as_list(f.launch_host(ins, len(ins[0]), table=extra["table"]))
        else:
            got = _as_list(f(*ins))
        s = f.stats(raise_on_device_error=True)
    _check(name, got, outs)
    assert s["threads"] == len(ins[0])


def test_plain_block_sizes(golden):
    ins, outs = golden("collatz_u64")
    for bs in (32, 128, 512, 1024):
        with api.Function("collatz_u64", len(ins[0]), "plain", block_size=bs) as f:
            _check("collatz_u64", _as_list(f(*ins)), outs)


@pytest.mark.parametrize("mode", ["plain", "regroup"])
def test_instruction_count_equals_oracle(mode, golden):
    ins, outs = golden("collatz_u64")
    (_,), counts = O.Interp("collatz_u64").run(ins, count_instr=True)
    with api.Function("collatz_u64", len(ins[0]), mode, profile=True) as f:
        f(*ins)
        s = f.stats(raise_on_device_error=True)
    assert s["thread_instr"] == int(counts.sum())
    assert 0.0 < s["lane_efficiency"] <= 1.0


def test_fib_config0_full_size():
    """2^20 threads, n uniform in [0, 93]: bit-exact against the numpy
    restatement of Loom's val_fib (programs.hpp:353-368)."""
    n = O.uniform_int(11, 1 << 20, 0, 93)
    want = O.val_fib(n)
    for mode in ("plain", "regroup"):
        with api.Function("fib_u64", len(n), mode) as f:
            got = f(n)
            f.stats(raise_on_device_error=True)
        assert np.array_equal(got, want), mode


def test_collatz_large_plain_equals_regroup_and_oracle_sample():
    """2^22 threads: both engines agree on every thread; a seeded sample
    matches the C oracle; known stopping times hold."""
    n = O.uniform_int(12, 1 << 22, 1, (1 << 32) - 1)
    n[:4] = [27, 97, 837799, 1]
    with api.Function("collatz_u64", len(n), "plain") as f:
        a = f(n)
    with api.Function("collatz_u64", len(n), "regroup", population=1 << 18) as f:
        b = f(n)
        s = f.stats(raise_on_device_error=True)
    assert np.array_equal(a, b)
    assert a[:4].tolist() == [111, 118, 524, 0]
    idx = O.uniform_int(13, 4096, 0, len(n) - 1).astype(np.int64)
    (want,) = O.Interp("collatz_u64").run([n[idx]])
    assert np.array_equal(a[idx], want)
    assert s["threads"] == len(n)


def test_iota_input_column():
    """A NULL input column feeds the thread index (no input traffic)."""
    with api.Function("collatz_u64", 5000, "regroup") as f:
        got = f(None, n=5000)
    assert np.array_equal(got, O.val_collatz(np.arange(5000, dtype=np.uint64)))


@pytest.mark.parametrize("mode", ["plain", "regroup"])
def test_step_guard_ends_a_runaway_thread(mode):
    """fib(2^64 - 1) never halts; the step guard ends it with a status bit
    instead of hanging the GPU, the other threads finish, and the handle
    stays usable."""
    n = np.arange(64, dtype=np.uint64)
    n[5] = np.uint64(2**64 - 1)
    with api.Function("fib_u64", len(n), mode, max_steps=2000, period=16) as f:
        with pytest.raises(api.LoomError) as e:
            f(n)
        assert e.value.code == api.ERR_DEVICE
        assert f.stats()["status"] & api.STATUS_STEP_LIMIT
        good = np.delete(np.arange(64), 5)
        f.reset_stats()
        m = n.copy()
        m[5] = 7
        got = f(m)
        assert np.array_equal(got, O.val_fib(m))


def test_barrier_wait_is_bounded():
    """Fault injection: the grid barrier waits for CTAs that do not exist;
    its bounded wait runs out, the status word says so, and the next launch
    on the same handle is correct."""
    n = O.uniform_int(3, 4096, 0, 93)
    with api.Function("fib_u64", len(n), "regroup", fault_phantom_ctas=1, barrier_spins=20000) as f:
        with pytest.raises(api.LoomError):
            f(n)
        assert f.stats()["status"] & api.STATUS_BARRIER_TIMEOUT
        f.set_opts("regroup")
        f.reset_stats()
        assert np.array_equal(f(n), O.val_fib(n))


def test_run_device_with_torch_columns():
    import torch

    n = O.uniform_int(21, 100000, 1, 1 << 20)
    d_in = torch.from_numpy(n.view(np.int64)).cuda()
    d_out = torch.empty(len(n), dtype=torch.int32, device="cuda")
    with api.Function("collatz_u64", 0, "regroup") as f:
        f.run_device([d_in], [d_out], len(n), stream=torch.cuda.current_stream())
        torch.cuda.synchronize()
        f.sync()
    got = d_out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, O.val_collatz(n))


def test_graph_replay_equals_direct_launch():
    """opts.graph: the regrouping launch sequence is captured once and
    replayed while the arguments stay the same; new arguments re-capture."""
    import torch

    x = O.uniform_int(31, 50000, 1, 1 << 32)
    d_x = torch.from_numpy(x.view(np.int64)).cuda()
    outs = [torch.empty(len(x), dtype=torch.int32, device="cuda") for _ in range(2)]
    with api.Function("collatz_u64", 0, "regroup", graph=True) as f:
        for _ in range(3):
            f.run_device([d_x], [outs[0]], len(x))
            f.sync()
        s = f.stats(raise_on_device_error=True)
        assert (s["graph_captures"], s["graph_launches"]) == (1, 3)
        f.run_device([d_x], [outs[1]], len(x))  # another output column: new graph
        f.sync()
        s = f.stats(raise_on_device_error=True)
        assert (s["graph_captures"], s["graph_launches"]) == (2, 4)
    want = O.val_collatz(x)
    for o in outs:
        assert np.array_equal(o.cpu().numpy().view(np.uint32), want)


@pytest.mark.parametrize("mode", ["plain", "regroup"])
def test_block_stats_add_up(mode, golden):
    """Per-block counters of a profiled launch sum to the launch totals, and
    every thread executes exactly the oracle's instruction count."""
    ins, _ = golden("fib_u64")
    with api.Function("fib_u64", len(ins[0]), mode, profile=True) as f:
        f(*ins)
        s = f.stats(raise_on_device_error=True)
        blocks = f.block_stats()
    assert sum(b["thread_instr"] for b in blocks) == s["thread_instr"]
    assert sum(b["warp_instr"] for b in blocks) == s["warp_instr"]
    _, cnt = O.Interp("fib_u64").run(ins, count_instr=True)
    assert s["thread_instr"] == int(cnt.sum())
    assert all(b["warp_instr"] * 32 >= b["thread_instr"] for b in blocks)


def test_loom_pt2_engines_agree_bit_for_bit(golden):
    """Where the scalar backend is matched within ULP_TOLERANCE (libm sin and
    cos), the two engines still agree with each other exactly."""
    ins, _ = golden("pt2_const_40")
    got = {}
    for mode in ("plain", "regroup"):
        with api.Function("pt2_const_40", len(ins[0]), mode) as f:
            got[mode] = _as_list(f(*ins))
            f.stats(raise_on_device_error=True)
    for a, b in zip(got["plain"], got["regroup"]):
        assert np.array_equal(_bits(a), _bits(b))


def test_headless_render_writes_a_png(tmp_path):
    """The render command traces a small Cornell image on the device and
    writes it as a PNG; both engines give the same pixels."""
    from loom_b200 import render as Rd
    from loom_b200 import scenes as S

    req = S.cornell_request(32, 24, 4, seed=3)
    a = Rd.render(req, "regroup")
    b = Rd.render(req, "plain")
    assert a.shape == (32 * 24, 3) and np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert float(a.mean()) > 0.0
    out = tmp_path / "c.png"
    Rd.main(["--out", str(out), "--width", "32", "--height", "24", "--spp", "4"])
    assert out.read_bytes()[:8] == b"\x89PNG\r\n\x1a\n"
