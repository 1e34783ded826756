"""State inspection: where the regrouping engine's threads wait, and with what.

Loom's inspector (src/vm/dbg.hpp:918-933 `print_state`, 1143 `inspect`)
steps one thread on the CPU and prints its PC label and registers per step.
On the B200 the interesting state is the regrouping engine's: the work
queues in which threads wait at a block entry with their live registers.
A launch whose round limit (`max_steps` of the regrouping engine) runs out
leaves its threads parked there; this module reads them back and prints
them one row per thread, PC label first, as `print_state` does:

    python -m loom_b200.inspector collatz_u64 --n 65536 --rounds 1 --period 4
    python -m loom_b200.inspector sphere_pt_f32 --n 16384 --rounds 2

Integer inputs are drawn uniformly from [--lo, --hi), float inputs from
[0, 1), with a fixed seed; `sphere_pt_f32` traces the Cornell box (one
request, thread index = pixel sample).
"""

from __future__ import annotations

import argparse
from typing import Dict, List, Sequence

import numpy as np

from . import api


def label(block: int, context: int) -> str:
    """The PC label of a queue: its block, and for a subroutine block the
    caller's context."""
    if block == 0:
        base = "START"
    else:
        base = f"B{block}"
    return base if context < 0 else f"{base}<{context}>"


def _fmt(v) -> str:
    if isinstance(v, (np.floating, float)):
        return f"{float(v):.6g}"
    return str(int(v))


def format_parked(parked: Sequence[Dict], rows: int = 8, width: int = 12) -> str:
    """Text table of `Function.parked()`: per queue a header with its label
    and row count, then up to `rows` threads (thread index, then each live
    register)."""
    out: List[str] = []
    total = sum(q["rows"] for q in parked)
    out.append(f"{total} parked threads in {len(parked)} queues")
    for q in parked:
        names = list(q["regs"])
        out.append("")
        out.append(f"{label(q['block'], q['context'])}: {q['rows']} threads")
        out.append("".join(c.rjust(width) for c in ["tid", *names]))
        for i in range(min(rows, q["rows"])):
            vals = [_fmt(q["tid"][i])] + [_fmt(q["regs"][n][i]) for n in names]
            out.append("".join(v.rjust(width) for v in vals))
    return "\n".join(out)


def _inputs(kernel: str, n: int, lo: int, hi: int, seed: int):
    info = api.info(kernel)
    rng = np.random.default_rng(seed)
    cols = []
    for _, t in info.inputs:
        dt = np.dtype(api.NP_TYPE[t])
        if dt.kind == "f":
            cols.append(rng.random(n).astype(dt))
        else:
            top = min(hi, int(np.iinfo(dt).max) + 1)
            cols.append(rng.integers(lo, max(lo + 1, top), size=n, dtype=np.int64).astype(dt))
    return cols


def run(kernel: str, n: int, rounds: int, period: int, population: int, lo: int, hi: int, seed: int):
    """One regrouping launch limited to `rounds` rounds; returns the handle's
    parked rows and its stats."""
    opts = dict(max_steps=rounds, period=period, population=population, prefetch=False)
    with api.Function(kernel, n, "regroup", **opts) as f:
        try:
            if kernel == "sphere_pt_f32":
                from . import scenes as S

                side = max(1, int(np.sqrt(n / 4)))
                req = S.cornell_request(side, side, 4, seed=seed)
                table, starts = S.pack([req])
                f.launch_host([api.Instance(), api.LocalIota()], req.threads, instance_starts=starts, table=table)
            else:
                f(*_inputs(kernel, n, lo, hi, seed))
        except api.LoomError as e:
            if e.code != api.ERR_DEVICE:
                raise
        st = f.stats()
        return f.parked(), st


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("kernel")
    ap.add_argument("--n", type=int, default=1 << 16, help="threads")
    ap.add_argument("--rounds", type=int, default=1, help="rounds of the megakernel before it stops")
    ap.add_argument("--period", type=int, default=16, help="block steps of a tile per round")
    ap.add_argument("--population", type=int, default=1 << 14, help="threads in flight")
    ap.add_argument("--lo", type=int, default=1)
    ap.add_argument("--hi", type=int, default=1 << 20)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--rows", type=int, default=8, help="rows printed per queue")
    a = ap.parse_args(argv)
    parked, st = run(a.kernel, a.n, a.rounds, a.period, a.population, a.lo, a.hi, a.seed)
    print(f"{a.kernel}: {st['rounds']} rounds, {st['threads']} threads finished, status {st['status']:#x}")
    print(format_parked(parked, a.rows))


if __name__ == "__main__":
    main()
