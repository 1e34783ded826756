"""State inspection on the GPU: a regrouping launch stopped by its round
limit leaves threads parked in the work queues; the rows read back are the
exact states of those threads (checked against the Collatz map run on the
host for the recorded number of steps), no thread is both parked and
finished, and a launch that finishes leaves nothing parked."""

import numpy as np
import pytest

from loom_b200 import api
from loom_b200 import inspector as I

pytestmark = pytest.mark.gpu

SENTINEL = 0xFFFFFFFF


def collatz_steps(x, s):
    """The Collatz map applied s[i] times to x[i] (host, uint64)."""
    x = x.astype(np.uint64).copy()
    s = s.astype(np.int64)
    for i in range(int(s.max()) if len(s) else 0):
        m = s > i
        v = x[m]
        x[m] = np.where(v & np.uint64(1), np.uint64(3) * v + np.uint64(1), v >> np.uint64(1))
    return x


def reference_steps(x):
    x = x.astype(np.uint64).copy()
    steps = np.zeros(len(x), dtype=np.uint32)
    live = x > 1
    while live.any():
        v = x[live]
        x[live] = np.where(v & np.uint64(1), np.uint64(3) * v + np.uint64(1), v >> np.uint64(1))
        steps[live] += 1
        live = x > 1
    return steps


def test_parked_collatz_rows_are_exact_states():
    import torch

    n = 1 << 16
    x = np.random.default_rng(11).integers(1, 1 << 32, size=n, dtype=np.uint64)
    d_in = torch.from_numpy(x.view(np.int64)).cuda()
    d_out = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    opts = dict(max_steps=1, period=8, population=1 << 13, prefetch=False)
    with api.Function("collatz_u64", n, "regroup", **opts) as f:
        f.launch_device([d_in], [d_out], n)
        with pytest.raises(api.LoomError) as e:
            f.sync()
        assert e.value.code == api.ERR_DEVICE
        st = f.stats()
        assert st["status"] & 1  # the round limit ran out
        parked = f.parked()
    out = d_out.cpu().numpy().view(np.uint32)
    finished = np.flatnonzero(out != SENTINEL)
    assert len(finished) == st["threads"]
    assert np.array_equal(out[finished], reference_steps(x[finished]))

    assert parked, "the round limit left no thread parked"
    seen = []
    for q in parked:
        tid = q["tid"].astype(np.int64)
        assert (tid < n).all()
        seen.append(tid)
        if q["block"] == 0:
            assert np.array_equal(q["regs"]["n"], x[tid])
        else:
            assert q["block"] == 1
            got = q["regs"]["n"]
            assert np.array_equal(got, collatz_steps(x[tid], q["regs"]["steps"]))
    seen = np.concatenate(seen)
    assert len(np.unique(seen)) == len(seen), "a thread parked twice"
    assert not np.isin(seen, finished).any(), "a finished thread is also parked"
    assert len(seen) + len(finished) <= n


def test_a_finished_launch_leaves_nothing_parked():
    n = 1 << 14
    x = np.random.default_rng(5).integers(1, 1 << 20, size=n, dtype=np.uint64)
    with api.Function("collatz_u64", n, "regroup", period=8, population=1 << 12) as f:
        steps = f(x)
        assert f.parked() == []
    assert np.array_equal(steps, reference_steps(x))
    with api.Function("collatz_u64", n, "plain") as f:
        f(x)
        assert f.parked() == []


def test_inspector_on_the_path_tracer():
    parked, st = I.run("sphere_pt_f32", 1 << 14, rounds=2, period=16, population=1 << 12, lo=0, hi=1, seed=1)
    assert st["status"] & 1
    assert parked
    tids = np.concatenate([q["tid"] for q in parked]).astype(np.int64)
    assert len(np.unique(tids)) == len(tids)
    assert (tids < (1 << 14)).all()
    qs = api.queues("sphere_pt_f32")
    for q in parked:
        lay = qs[q["queue"]]
        assert q["block"] == lay["block"] and q["context"] == lay["context"]
        assert list(q["regs"]) == [c[1] for c in lay["cols"]]
    text = I.format_parked(parked, rows=2)
    assert text.startswith(f"{len(tids)} parked threads")
