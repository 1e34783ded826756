"""A request loop over several kernels: one continuous-batching server
(loom_b200_server_*) per kernel, all on one CUDA stream, stepped in turn.

Each ``step`` gives every server that has work one slice of its
regrouping megakernel; a request admitted by a server joins the threads of
that server's requests in flight.  Completions come back as
``(kind, ticket)`` pairs; ``result`` hands out the outputs.
"""

from __future__ import annotations

from typing import Dict, List, Tuple

from . import api


class Pool:
    def __init__(self, servers: Dict[str, api.Server]):
        self.servers = dict(servers)
        self._work = {k: 0 for k in self.servers}  # submitted, not completed

    def submit(self, kind: str, n: int, **request) -> Tuple[str, int]:
        t = self.servers[kind].submit(n, **request)
        self._work[kind] += 1
        return kind, t

    def busy(self) -> bool:
        return any(self._work.values())

    def step(self) -> List[Tuple[str, int]]:
        done = []
        for k, srv in self.servers.items():
            if self._work[k]:
                for t in srv.step():
                    done.append((k, t))
                    self._work[k] -= 1
        return done

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
