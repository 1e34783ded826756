"""A request loop over several kernels: one continuous-batching server
(loom_b200_server_*) per kernel, each on its own CUDA stream.

Each ``step`` gives every server that has work one slice of its
regrouping megakernel; a request admitted by a server joins the threads of
that server's requests in flight.  When several servers have work, their
slices are started together (``Server.launch`` with the CTAs per SM of
``shared_ctas``, so that the cooperative grids fit on the SMs side by side)
and then completed, so the kernels of different requests run on the GPU at
the same time, as Loom's mp::Shop runs several kernels' streams at once
(src/vm/mp.hpp:316-385).  Servers created with one ``api.Budget`` admit
requests against that shared device-memory budget.  Completions come back
as ``(kind, ticket)`` pairs; ``result`` hands out the outputs.  Requests
cancelled by ``cancel`` or by a server's watchdog (``timeout``) come back
from ``failures`` as ``(kind, ticket, code)``.
"""

from __future__ import annotations

from typing import Dict, List, Optional, Tuple

from . import api


class Pool:
    def __init__(self, servers: Dict[str, api.Server], timeout: float = 0.0,
                 shared_ctas: Optional[Dict[str, int]] = None):
        self.servers = dict(servers)
        # CTAs per SM of each server's slice while several servers run (None:
        # one server after the other)
        self.shared_ctas = shared_ctas
        self.slice_ns = 0  # device time of the slices, summed over servers
        self.union_ns = 0  # time at least one slice ran
        self._work = {k: 0 for k in self.servers}  # submitted, not completed
        self._failed: List[Tuple[str, int, int]] = []
        if timeout:
            for srv in self.servers.values():
                srv.set_timeout(timeout)

    def submit(self, kind: str, n: int, **request) -> Tuple[str, int]:
        t = self.servers[kind].submit(n, **request)
        self._work[kind] += 1
        return kind, t

    def busy(self) -> bool:
        return any(self._work.values())

    def step(self) -> List[Tuple[str, int]]:
        done = []
        busy = [k for k, srv in self.servers.items() if self._work[k]]
        together = bool(self.shared_ctas) and len(busy) > 1
        if together:
            for k in busy:
                self.servers[k].launch(self.shared_ctas.get(k, 1))
        spans = []
        for k in busy:
            srv = self.servers[k]
            slices = srv.stats()["slices"]
            for t in srv.step():
                done.append((k, t))
                self._work[k] -= 1
            st = srv.stats()
            if st["slices"] > slices and st["slice_t1_ns"] > st["slice_t0_ns"]:
                spans.append((st["slice_t0_ns"], st["slice_t1_ns"]))
            self._collect(k, srv)
        self._account(spans)
        return done

    def _account(self, spans) -> None:
        """Adds this step's slice intervals (global-timer ns) to the device
        time of the slices (their sum) and to the time any slice ran (their
        union): sum / union above 1 means slices of different kernels ran on
        the GPU at the same time."""
        if not spans:
            return
        self.slice_ns += sum(b - a for a, b in spans)
        union, end = 0, 0
        for a, b in sorted(spans):
            a = max(a, end)
            if b > a:
                union += b - a
                end = b
        self.union_ns += union

    def overlap(self) -> float:
        """Summed slice time over the time any slice ran (1.0: no overlap)."""
        return self.slice_ns / self.union_ns if self.union_ns else 1.0

    def cancel(self, kind: str, ticket: int) -> bool:
        ok = self.servers[kind].cancel(ticket)
        self._collect(kind, self.servers[kind])
        return ok

    def failures(self) -> List[Tuple[str, int, int]]:
        """(kind, ticket, code) of the requests that ended without
        completing since the last call."""
        out, self._failed = self._failed, []
        return out

    def _collect(self, kind: str, srv: api.Server) -> None:
        for t, code in srv.failed():
            self._failed.append((kind, t, code))
            self._work[kind] -= 1

    def result(self, kind: str, ticket: int):
        return self.servers[kind].result(ticket)

    def stats(self) -> Dict[str, Dict[str, int]]:
        return {k: s.stats() for k, s in self.servers.items()}

    def close(self) -> None:
        for s in self.servers.values():
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
