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
