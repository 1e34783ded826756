"""The host-facing paths around the engines (needs a GPU): images as
per-group means on the device, the pipelined host launch, register caps of
the megakernel and the queue-free form of schedule 2.

Every result is compared bit for bit with Loom bse's outputs (the golden
fixtures) or with a host restatement of the same arithmetic (the per-pixel
mean of scenes.pixel_average: samples summed in order in float32, divided
by the sample count).
"""

import numpy as np
import pytest

from loom_b200 import api
from loom_b200 import scenes as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def _instance_means(outs, starts, spp):
    """Per-request images from per-sample outputs, requests in order."""
    rows = []
    for i in range(len(spp)):
        a, b = int(starts[i]), int(starts[i + 1])
        rows.append(S.pixel_average([np.asarray(o)[a:b] for o in outs], int(spp[i])))
    return np.concatenate(rows, axis=0)


def _fixture_spp(extra):
    table = extra["table"]
    n_inst = len(extra["starts"]) - 1
    return np.array([1 << int(table[i * S.HEADER_WORDS + 2]) for i in range(n_inst)], dtype=np.uint32)


@pytest.mark.parametrize("mode", ["plain", "regroup"])
def test_launch_host_mean_equals_pixel_average_of_bse(mode, golden, golden_extra):
    """The batched path-tracing fixture: every request's image through
    loom_b200_launch_host_mean equals the per-pixel means of bse's
    per-sample outputs."""
    ins, outs = golden("sphere_pt_f32")
    extra = golden_extra("sphere_pt_f32")
    n = len(ins[0])
    spp = _fixture_spp(extra)
    want = _instance_means(outs, extra["starts"], spp)
    with api.Function("sphere_pt_f32", n, mode) as f:
        got = f.launch_host_mean([api.Instance(), api.LocalIota()], n, instance_group=spp,
                                 instance_starts=extra["starts"], table=extra["table"])
        f.stats(raise_on_device_error=True)
    got = np.stack(got, axis=1)
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_group_mean_device_column():
    """loom_b200_group_mean on a device column against the host mean, for
    groups of 1, 4, 64 and 7 (not a power of two)."""
    import torch

    rng = np.random.default_rng(4)
    for g in (1, 4, 64, 7):
        rows = 10_001
        x = rng.standard_normal(rows * g).astype(np.float32) * 1e3
        d_x = torch.from_numpy(x).cuda()
        d_y = torch.empty(rows, dtype=torch.float32, device="cuda")
        api.group_mean(d_x, d_y, rows, g)
        torch.cuda.synchronize()
        want = S.pixel_average([x], g)[:, 0]
        assert np.array_equal(d_y.cpu().numpy().view(np.uint32), want.view(np.uint32)), g


def test_launch_host_mean_rejects_ragged_groups(golden_extra):
    extra = golden_extra("sphere_pt_f32")
    n = int(extra["starts"][-1])
    with api.Function("sphere_pt_f32", n, "regroup") as f:
        with pytest.raises(api.LoomError) as e:
            # 6144 threads are no multiple of 5
            f.launch_host_mean([api.Instance(), api.LocalIota()], n, group=5,
                               instance_starts=extra["starts"], table=extra["table"])
        assert e.value.code == api.ERR_INVALID
    with api.Function("collatz_u64", 64, "regroup") as f:
        with pytest.raises(api.LoomError):  # integer outputs have no mean
            f.launch_host_mean([np.arange(64, dtype=np.uint64)], 64, group=4)


@pytest.mark.parametrize("chunks", [1, 3, 8])
@pytest.mark.parametrize("mode", ["plain", "regroup"])
def test_pipelined_host_launch(mode, chunks):
    """A host launch split into ranges whose copies overlap the kernels
    equals one range and the validator, for ranges that do not divide n."""
    n = 300_007
    x = O.uniform_int(21, n, 1, (1 << 32) - 1)
    with api.Function("collatz_u64", n, mode, host_chunks=chunks) as f:
        got = f(x)
        s = f.stats(raise_on_device_error=True)
    assert s["threads"] == n
    idx = O.uniform_int(22, 4096, 0, n - 1).astype(np.int64)
    assert np.array_equal(got[idx], O.val_collatz(x[idx]))
    with api.Function("collatz_u64", n, mode) as f:
        assert np.array_equal(f(x), got)


def test_pipelined_host_launch_iota_and_instances(golden, golden_extra):
    """Ranges start at thread ids other than 0: the iota form, the instance
    forms and the table follow the global thread id."""
    ins, outs = golden("sphere_pt_f32")
    extra = golden_extra("sphere_pt_f32")
    n = len(ins[0])
    with api.Function("sphere_pt_f32", n, "regroup", host_chunks=5) as f:
        got = f.launch_host([api.Instance(), api.LocalIota()], n, instance_starts=extra["starts"],
                            table=extra["table"])
        f.stats(raise_on_device_error=True)
    for g, w in zip(got, outs):
        assert np.array_equal(_bits(g), _bits(w))
    with api.Function("collatz_u64", 5000, "plain", host_chunks=4) as f:
        got = f(None, n=5000)
    assert np.array_equal(got, O.val_collatz(np.arange(5000, dtype=np.uint64)))


@pytest.mark.parametrize("name", ["sphere_pt_f32", "pt_const_40"])
def test_register_caps_keep_results(name, golden, golden_extra):
    """Every register cap compiled for the megakernel gives bse's outputs."""
    ins, outs = golden(name)
    extra = golden_extra(name)
    caps = api.reg_caps(name)
    assert len(caps) > 1
    for cap in caps:
        with api.Function(name, len(ins[0]), "regroup", max_regs=cap, schedule=2,
                          period=api.PERIOD_UNBOUNDED, burst=2) as f:
            if "table" in extra:
                got = f.launch_host(ins, len(ins[0]), table=extra["table"])
            else:
                got = f(*ins)
            f.stats(raise_on_device_error=True)
        got = list(got) if isinstance(got, tuple) else [got]
        for g, w in zip(got, outs):
            assert np.array_equal(_bits(g), _bits(w)), cap


def test_register_cap_not_compiled_is_refused():
    assert 72 not in api.reg_caps("collatz_u64")
    with api.Function("collatz_u64", 64, "regroup", max_regs=72) as f:
        with pytest.raises(api.LoomError) as e:
            f(np.arange(64, dtype=np.uint64))
        assert e.value.code == api.ERR_INVALID


def test_never_parking_form_holds_no_queue_state():
    """Schedule 2 without a period limit runs one round and reserves one
    tile per queue: its device memory is a few KB beyond the columns, while
    a parking form of the same launch reserves queue state per thread in
    flight."""
    n = 1 << 20
    x = O.uniform_int(23, n, 1, (1 << 32) - 1)
    d = {}
    for name, opts in (("never", dict(schedule=2, period=api.PERIOD_UNBOUNDED, burst=2)),
                       ("parks", dict(population=1 << 18))):
        with api.Function("collatz_u64", n, "regroup", **opts) as f:
            got = f(x)
            s = f.stats(raise_on_device_error=True)
            d[name] = (f.device_bytes(), s["rounds"], s["parks"], got)
    cols = n * (8 + 4)
    assert d["never"][0] - cols < (64 << 10)
    assert d["never"][1] == 1 and d["never"][2] == 0
    assert d["parks"][0] - cols > (1 << 18) * 8
    assert np.array_equal(d["never"][3], d["parks"][3])


def test_group_mean_tiles_and_fallbacks():
    """The means' shared-memory tiles (groups of 8, 16 and 32 here) and
    their fallbacks: a column that does not start on a 16-byte boundary and
    an f64 column, each against the host mean in order."""
    import torch

    rng = np.random.default_rng(6)
    rows = 1000
    for g, dtype, shift in ((8, np.float32, 0), (16, np.float32, 0), (32, np.float32, 0), (16, np.float32, 1),
                            (16, np.float64, 0)):
        x = (rng.standard_normal(rows * g + shift) * 1e3).astype(dtype)
        d_x = torch.from_numpy(x).cuda()
        d_y = torch.empty(rows, dtype=torch.from_numpy(x[:1]).dtype, device="cuda")
        api.group_mean(d_x[shift:], d_y, rows, g)
        torch.cuda.synchronize()
        want = _ordered_means(x[shift:], g)
        assert np.array_equal(d_y.cpu().numpy(), want), (g, dtype, shift)


def _ordered_means(x, g):
    """Means of consecutive groups of g, summed in order in x's type."""
    s = np.asarray(x).reshape(-1, g)
    acc = np.zeros(s.shape[0], dtype=s.dtype)
    for j in range(g):
        acc = acc + s[:, j]
    return acc / s.dtype.type(g)


def test_launch_host_mean_warps_across_instances():
    """Instances whose rows do not fill whole warps, with groups from 1 to 64:
    the warps whose 32 rows straddle two instances read their rows lane by
    lane, the others through the shared-memory tile; every mean equals the
    in-order mean of the engine's own per-thread outputs."""
    rng = np.random.default_rng(8)
    groups = np.array([4, 16, 1, 64, 8, 2, 32, 4], dtype=np.uint32)
    rows = np.array([33, 5, 70, 3, 41, 17, 9, 64], dtype=np.int64)
    starts = np.concatenate([[0], np.cumsum(groups.astype(np.int64) * rows)]).astype(np.uint64)
    n = int(starts[-1])
    x = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    with api.Function("canonical_f32", n, "plain") as f:
        per = f.launch_host([x], n)  # one output: the array itself
        (got,) = f.launch_host_mean([x], n, instance_group=groups, instance_starts=starts)
        f.stats(raise_on_device_error=True)
    want = np.concatenate([_ordered_means(per[int(starts[i]):int(starts[i + 1])], int(groups[i]))
                           for i in range(len(groups))])
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
