"""Serving (loom_b200_server_*): continuous batching on the regrouping
engine (needs a GPU).

A result must not depend on what else was in flight: every request's
outputs are compared bit for bit with the same request run alone and with
the oracle, while the column rings wrap many times, slices end after one
round, and requests arrive while others run.
"""

import numpy as np
import pytest

from loom_b200 import api
from loom_b200 import scenes as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _drain(srv, pending, results, max_steps=100000):
    for _ in range(max_steps):
        if not pending:
            return
        for t in srv.step():
            results[t] = srv.result(t)
            pending.discard(t)
        assert srv.stats()["status"] == 0
    raise AssertionError(f"{len(pending)} requests still pending after {max_steps} slices")


def test_collatz_requests_through_wrapping_rings():
    rng = np.random.default_rng(11)
    sizes = rng.integers(1, 6000, size=60)
    reqs = [O.uniform_int(100 + i, int(n), 1, 1 << 32) for i, n in enumerate(sizes)]
    results = {}
    with api.Server("collatz_u64", ring_threads=1 << 14, max_requests=16, slice_rounds=1, population=2048, period=256) as srv:
        tickets = {srv.submit(len(x), [x]): i for i, x in enumerate(reqs)}
        _drain(srv, set(tickets), results)
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["threads"] == int(sizes.sum())
    assert st["slices"] > 10  # the rings (2^14 entries) wrapped many times
    for t, i in tickets.items():
        assert np.array_equal(results[t], O.val_collatz(reqs[i])), f"request {i}"


def _small_scene_requests(k, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        r = S.random_request(rng, seed=1000 + i)
        r.width = r.height = int(rng.choice([8, 16, 24]))
        r.spp = int(rng.choice([1, 4, 16]))
        out.append(r)
    return out


def _pt_server(**kw):
    return api.Server(
        "sphere_pt_f32",
        ring_threads=1 << 15,
        max_requests=8,
        forms=["instance", "local_iota"],
        header_words=S.HEADER_WORDS,
        reloc_word=4,
        table_words=1 << 14,
        **kw,
    )


def test_path_tracer_requests_alone_and_in_the_mix():
    reqs = _small_scene_requests(10, 5)
    words = [S.request_words(r) for r in reqs]

    alone = []
    with _pt_server(slice_rounds=2, burst=4, utr_lanes=8) as srv:
        for r, (h, b) in zip(reqs, words):
            t = srv.submit(r.threads, header=h, body=b)
            res = {}
            _drain(srv, {t}, res)
            alone.append(res[t])

    mixed = {}
    with _pt_server(slice_rounds=1, burst=4, utr_lanes=8, population=1024) as srv:
        # arrivals while others run: two up front, then one per slice
        order = list(range(len(reqs)))
        tickets = {}
        pending = set()
        for i in order[:2]:
            h, b = words[i]
            t = srv.submit(reqs[i].threads, header=h, body=b)
            tickets[t] = i
            pending.add(t)
        for i in order[2:]:
            for t in srv.step():
                mixed[tickets[t]] = srv.result(t)
                pending.discard(t)
            h, b = words[i]
            t = srv.submit(reqs[i].threads, header=h, body=b)
            tickets[t] = i
            pending.add(t)
        res = {}
        _drain(srv, pending, res)
        for t, v in res.items():
            mixed[tickets[t]] = v
        assert srv.stats()["status"] == 0

    # the same requests as one batched launch (instance offsets on the device)
    table, starts = S.pack(reqs)
    n = int(starts[-1])
    with api.Function("sphere_pt_f32", n, "regroup") as f:
        batch = f.launch_host([api.Instance(), api.LocalIota()], n, instance_starts=starts, table=table)

    for i, r in enumerate(reqs):
        lo, hi = int(starts[i]), int(starts[i + 1])
        for c in range(3):
            a = alone[i][c].view(np.uint32)
            assert np.array_equal(a, mixed[i][c].view(np.uint32)), f"request {i}: alone != mixed"
            assert np.array_equal(a, batch[c][lo:hi].view(np.uint32)), f"request {i}: alone != batch"

    # and a sample against the oracle
    idx = np.sort(O.uniform_int(9, 64, 0, n - 1).astype(np.int64))
    ins = O.expand_inputs(["instance", "local_iota"], n, starts, ["u32", "u32"])
    want = O.Interp("sphere_pt_f32").run([a[idx] for a in ins], table=table)
    for c in range(3):
        assert np.array_equal(batch[c][idx].view(np.uint32), want[c].view(np.uint32))


def test_request_larger_than_the_ring_is_refused():
    with api.Server("collatz_u64", ring_threads=1 << 10, max_requests=4) as srv:
        with pytest.raises(api.LoomError) as e:
            srv.submit(2000, [np.ones(2000, dtype=np.uint64)])
        assert e.value.code == api.ERR_BUDGET


def _collatz_reqs(k, n, seed):
    return [O.uniform_int(seed + i, n, 1, 1 << 32) for i in range(k)]


def test_budget_defers_requests_until_bytes_free_up():
    """Admission by thread-state bytes: with a budget for two requests, the
    third waits until one completes; every result is still right and the
    budget comes back to zero."""
    info = api.info("collatz_u64")
    n = 4096
    per_request = n * (info.state_size + 8 + 4)  # state + input u64 + output u32
    budget = api.Budget(2 * per_request)
    reqs = _collatz_reqs(5, n, 300)
    results = {}
    with api.Server("collatz_u64", ring_threads=1 << 16, max_requests=16, slice_rounds=1, period=16,
                    population=1024, budget=budget) as srv:
        tickets = {srv.submit(n, [x]): i for i, x in enumerate(reqs)}
        # first slice: two admitted, three waiting for the budget
        for t in srv.step():
            results[t] = srv.result(t)
        st = srv.stats()
        assert st["admitted"] == 2 and st["budget_waits"] >= 1
        assert budget.used == 2 * per_request == st["held_bytes"]
        _drain(srv, set(tickets) - set(results), results)
        st = srv.stats()
    assert st["completed"] == 5 and st["held_bytes"] == 0 and budget.used == 0
    for t, i in tickets.items():
        assert np.array_equal(results[t], O.val_collatz(reqs[i]))


def test_request_larger_than_the_budget_is_refused():
    budget = api.Budget(1000)
    with api.Server("collatz_u64", ring_threads=1 << 12, max_requests=4, budget=budget) as srv:
        with pytest.raises(api.LoomError) as e:
            srv.submit(1000, [np.ones(1000, dtype=np.uint64)])
        assert e.value.code == api.ERR_BUDGET


def test_budget_shared_by_two_servers():
    """Two servers on one budget: what one holds, the other cannot admit."""
    info = api.info("collatz_u64")
    n = 2048
    per_request = n * (info.state_size + 8 + 4)
    budget = api.Budget(per_request)
    x, y = _collatz_reqs(2, n, 400)
    with api.Server("collatz_u64", ring_threads=1 << 14, max_requests=4, slice_rounds=1, period=8,
                    population=512, budget=budget) as a, \
         api.Server("collatz_u64", ring_threads=1 << 14, max_requests=4, slice_rounds=1, period=8,
                    population=512, budget=budget) as b:
        ta = a.submit(n, [x])
        tb = b.submit(n, [y])
        ra, rb = {}, {}
        done_a = a.step()
        assert budget.used == per_request  # a's request holds the whole budget
        b.step()
        assert b.stats()["admitted"] == 0 and b.stats()["budget_waits"] == 1
        for t in done_a:
            ra[t] = a.result(t)
        _drain(a, {ta} - set(ra), ra)
        assert budget.used == 0
        _drain(b, {tb}, rb)
    assert np.array_equal(ra[ta], O.val_collatz(x)) and np.array_equal(rb[tb], O.val_collatz(y))


def test_cancel_queued_and_in_flight_requests():
    """A queued request leaves at once; one in flight is dropped when its
    threads have finished (its outputs are not copied out); both come back
    once from failed() with ERR_CANCELLED, and the others complete."""
    reqs = _collatz_reqs(4, 3000, 500)
    outs = [np.full(3000, 0xFFFFFFFF, dtype=np.uint32) for _ in reqs]
    with api.Server("collatz_u64", ring_threads=1 << 14, max_requests=2, slice_rounds=1, period=4,
                    population=256) as srv:
        t = [srv.submit(3000, [x], outputs=[o]) for x, o in zip(reqs, outs)]
        srv.step()  # two admitted (two slots), two queued
        st = srv.stats()
        assert st["in_flight"] == 2 and st["queued"] == 2
        assert srv.cancel(t[3])  # queued
        assert srv.cancel(t[0])  # in flight
        assert not srv.cancel(t[0])  # once
        res = {}
        _drain(srv, {t[1], t[2]}, res)
        failed = dict(srv.failed())
        for _ in range(50):  # the in-flight one is reported after its threads finished
            if t[0] in failed:
                break
            srv.step()
            failed.update(dict(srv.failed()))
    assert failed == {t[3]: api.ERR_CANCELLED, t[0]: api.ERR_CANCELLED}
    assert (outs[0] == 0xFFFFFFFF).all() and (outs[3] == 0xFFFFFFFF).all()
    for i in (1, 2):
        assert np.array_equal(res[t[i]], O.val_collatz(reqs[i]))


def test_watchdog_times_out_old_requests():
    """With a timeout, requests older than it are ended with ERR_TIMEOUT at
    the next step (the host-side watchdog); a new request after that
    completes normally."""
    import time

    reqs = _collatz_reqs(3, 2000, 600)
    with api.Server("collatz_u64", ring_threads=1 << 14, max_requests=1, slice_rounds=1, period=2,
                    population=64) as srv:
        srv.set_timeout(0.05)
        ts = [srv.submit(2000, [x]) for x in reqs]
        time.sleep(0.1)
        srv.step()
        failed = dict(srv.failed())
        for _ in range(200):
            if len(failed) == 3:
                break
            srv.step()
            failed.update(dict(srv.failed()))
        assert failed == {t: api.ERR_TIMEOUT for t in ts}
        srv.set_timeout(0)
        x = O.uniform_int(700, 2000, 1, 1 << 32)
        t = srv.submit(2000, [x])
        res = {}
        _drain(srv, {t}, res)
    assert np.array_equal(res[t], O.val_collatz(x))


def test_pool_overlaps_servers_of_different_kernels():
    """A pool whose servers run on their own streams starts their slices
    together: on the GPU's global timer the slices of the two kernels run
    at the same time, and every result equals the validator's."""
    import torch

    from loom_b200 import serving

    streams = [torch.cuda.Stream() for _ in range(2)]
    cz = _collatz_reqs(6, 1 << 18, 800)
    fb = [O.uniform_int(900 + i, 1 << 18, 0, 93) for i in range(6)]
    pool = serving.Pool(
        {
            "collatz": api.Server("collatz_u64", ring_threads=1 << 20, max_requests=16, slice_rounds=2,
                                  block_size=256, population=1 << 18, stream=streams[0]),
            "fib": api.Server("fib_u64", ring_threads=1 << 20, max_requests=16, slice_rounds=2, block_size=256,
                              population=1 << 18, stream=streams[1]),
        },
        shared_ctas={"collatz": 1, "fib": 1},
    )
    keys = {}
    for i in range(6):
        keys[pool.submit("collatz", 1 << 18, inputs=[cz[i]])] = ("c", i)
        keys[pool.submit("fib", 1 << 18, inputs=[fb[i]])] = ("f", i)
    res = {}
    for _ in range(10000):
        if len(res) == len(keys):
            break
        for key in pool.step():
            res[key] = pool.result(*key)
    pool.close()
    assert len(res) == len(keys)
    for key, (kind, i) in keys.items():
        want = O.val_collatz(cz[i]) if kind == "c" else O.val_fib(fb[i])
        assert np.array_equal(res[key], want)
    # the slices' global-timer intervals intersect: summed slice time above
    # the time during which any slice ran
    assert pool.overlap() > 1.01, pool.overlap()
