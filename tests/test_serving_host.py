"""The request pool's bookkeeping on the host (loom_b200.serving.Pool) over
stand-in servers: completions and failures (cancelled or timed out) both
end a request's pending work, and the watchdog setting reaches every
server.  No GPU; the servers themselves are tested on a B200."""

from loom_b200.serving import Pool

CANCELLED, TIMEOUT = -8, -9


class FakeServer:
    def __init__(self, span=None, log=None):
        self.next = 0
        self.queued = []
        self.failed_q = []
        self.timeout = None
        self.slices = 0
        self.span = span  # (start, end) global-timer ns of every slice
        self.log = log if log is not None else []

    def stats(self):
        a, b = self.span or (0, 0)
        return {"slices": self.slices, "slice_t0_ns": a, "slice_t1_ns": b}

    def launch(self, ctas):
        self.log.append(("launch", self, ctas))

    def submit(self, n, **request):
        self.next += 1
        self.queued.append(self.next)
        return self.next

    def step(self):
        # completes the oldest request each step
        self.log.append(("step", self, None))
        if self.queued:
            self.slices += 1
        return [self.queued.pop(0)] if self.queued else []

    def cancel(self, ticket):
        if ticket in self.queued:
            self.queued.remove(ticket)
            self.failed_q.append((ticket, CANCELLED))
            return True
        return False

    def set_timeout(self, seconds):
        self.timeout = seconds

    def failed(self):
        out, self.failed_q = self.failed_q, []
        return out

    def expire_all(self):
        self.failed_q += [(t, TIMEOUT) for t in self.queued]
        self.queued = []

    def close(self):
        pass


def test_completions_and_cancellations_end_pending_work():
    a, b = FakeServer(), FakeServer()
    with Pool({"a": a, "b": b}) as pool:
        ta = [pool.submit("a", 10)[1] for _ in range(3)]
        tb = pool.submit("b", 5)[1]
        assert pool.busy()
        assert pool.cancel("a", ta[1])
        assert not pool.cancel("a", 99)
        assert pool.failures() == [("a", ta[1], CANCELLED)]
        done = []
        while pool.busy():
            done += pool.step()
        assert sorted(done) == sorted([("a", ta[0]), ("a", ta[2]), ("b", tb)])
        assert pool.failures() == []


def test_watchdog_failures_are_collected_by_step():
    a = FakeServer()
    with Pool({"a": a}, timeout=0.25) as pool:
        assert a.timeout == 0.25
        t = [pool.submit("a", 1)[1] for _ in range(2)]
        a.expire_all()
        assert pool.step() == []
        assert pool.failures() == [("a", t[0], TIMEOUT), ("a", t[1], TIMEOUT)]
        assert not pool.busy()


def test_busy_servers_start_their_slices_together():
    """With shared_ctas, a step with several busy servers starts every
    slice (launch with that server's CTAs per SM) before completing any; a
    step with one busy server just steps it.  The slices' global-timer
    intervals give the summed slice time and the time any slice ran."""
    log = []
    a = FakeServer(span=(100, 300), log=log)
    b = FakeServer(span=(200, 500), log=log)
    pool = Pool({"a": a, "b": b}, shared_ctas={"a": 1, "b": 2})
    pool.submit("a", 4)
    pool.submit("a", 4)
    pool.submit("b", 4)
    pool.step()
    assert [(e[0], e[1], e[2]) for e in log] == [("launch", a, 1), ("launch", b, 2), ("step", a, None), ("step", b, None)]
    assert (pool.slice_ns, pool.union_ns) == (200 + 300, 400)  # [100, 500] covered
    assert abs(pool.overlap() - 500 / 400) < 1e-12
    log.clear()
    pool.step()  # only a is busy now: no launch ahead of the step
    assert [e[0] for e in log] == ["step"]
    assert (pool.slice_ns, pool.union_ns) == (700, 600)
