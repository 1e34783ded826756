"""Autotuner of the regrouping engine's launch options.

The options that decide how well a kernel regroups depend on the kernel and
on its inputs: how many lanes must agree before a warp keeps running
(`utr_lanes`), how long a lane runs between votes (`burst`), when every live
lane runs along (`spread_lanes`), how many block steps a tile gets per round
(`period`), the threads in flight (`population`, which sizes every work
queue), the CTA size, the CTAs per SM, the megakernel's register cap
(`max_regs`, one of the caps compiled for the kernel: more registers per
thread mean fewer spills but fewer resident warps to hide latency) and
input prefetching.

`tune` runs a coordinate search: starting from a seed point it tries every
value of one option with the others fixed, keeps the fastest, moves to the
next option, and repeats the sweep until a pass brings less than 1 %.  With
several seeds (the stored point, the defaults with and without the cost
model) it searches from each and keeps the fastest point found.
Every point is timed on the device with CUDA events on the launching
stream (median of `reps` launches after one warm-up launch).  An optional
constraint (for instance a lane efficiency of at least some fraction,
measured by a counted launch) makes the points that miss it ineligible, so
the search returns the fastest point that meets it.  Results are
kept in `tuning.json` beside this module, per kernel and workload, and read
back by `tuned`.
"""

from __future__ import annotations

import json
import pathlib
import statistics
import time
from typing import Callable, Dict, List, Optional

HERE = pathlib.Path(__file__).resolve().parent
TUNING_FILE = HERE / "tuning.json"

SPACE: Dict[str, List] = {
    # between 8 and 16 the lane efficiency of schedule 2 on the path tracer
    # moves by a few per cent from one value to the next (when halted lanes
    # refill, against the loop's step count), so the grid is fine there
    "burst": [1, 2, 4, 8, 10, 12, 14, 16, 20, 24, 32, 64],
    "utr_lanes": [1, 4, 8, 12, 16, 20, 24],
    "spread_lanes": [1, 8, 16, 24, 33],
    # 0xffffffff: no period limit (schedule 2 then never parks)
    "period": [256, 1024, 4096, 16384, 65536, 1 << 20, 0xFFFFFFFF],
    "block_size": [128, 256, 512],
    "population": [1 << 18, 1 << 19, 1 << 20, 1 << 21, 1 << 22, 1 << 23],
    "ctas_per_sm": [0, 1, 2, 4],
    "prefetch": [True, False],
    "cost_model": [False, True],
    "schedule": [0, 1, 2, 3],
    # 0: the kernel's default cap; the others exist only for kernels large
    # enough to reach a cap (loom_b200_kernel_reg_caps), which the caller
    # passes as this option's values
    "max_regs": [0],
    # launches below this many threads run the plain engine: 0 never, 2^40
    # always (where the megakernel does not pay, the tuner may say so)
    "plain_below": [0, 1 << 40],
    # schedule 2: lanes a long block waits for (0: off)
    "defer_lanes": [0, 2, 4, 5, 6, 8, 12, 16, 24],
    # schedule 2: self-loop iterations per step (0: 1024)
    # (kernels of at most 300 instructions round to their compiled 16, 64
    # or 1024)
    "spin_iters": [0, 8, 16, 32, 64, 128],
    # schedule 2: halted lanes that end a burst early (0: off)
    "refill_lanes": [0, 1, 2, 4, 6, 8, 10, 12, 16],
}

DEFAULT = dict(burst=32, utr_lanes=16, spread_lanes=33, period=1024, block_size=256, population=0, ctas_per_sm=0, prefetch=True, cost_model=False, schedule=0, max_regs=0, plain_below=0, defer_lanes=0, spin_iters=0, refill_lanes=0)


def time_launch(fn: Callable[[], None], reps: int = 2) -> float:
    """Median device milliseconds of `fn` (launches on torch's current
    stream), after one warm-up call."""
    import torch

    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def tune(
    make_launch: Callable[[Dict], Callable[[], None]],
    n_threads: int,
    seed=None,
    space: Optional[Dict[str, List]] = None,
    passes: int = 2,
    reps: int = 2,
    budget_s: float = 600.0,
    log: Optional[Callable[[str], None]] = None,
    validate: Optional[Callable[[], None]] = None,
    constraint: Optional[Callable[[Dict], bool]] = None,
) -> Dict:
    """Coordinate search.  `make_launch(opts)` returns a no-argument callable
    that launches the workload once with those options; `validate()`, called
    after each timed point, raises when the launches set a device status;
    `constraint(opts)`, called after timing, returns False for a point that
    may not be chosen (it is recorded with "eligible": false).
    Returns {"best": opts, "ms": t, "points": [...]}."""
    space = dict(SPACE if space is None else space)
    seeds = [DEFAULT] if seed is None else (list(seed) if isinstance(seed, (list, tuple)) else [seed])
    cache: Dict[str, float] = {}
    points = []
    t_start = time.perf_counter()

    def measure(opts: Dict) -> float:
        key = json.dumps(opts, sort_keys=True)
        if key not in cache:
            if opts.get("population") and opts["population"] < 32:
                cache[key] = float("inf")
            else:
                ms = time_launch(make_launch(opts), reps)
                if validate:
                    validate()
                ok = constraint(opts) if constraint else True
                cache[key] = ms if ok else float("inf")
                pt = {"opts": dict(opts), "ms": round(ms, 4), "msamples_s": round(n_threads / ms / 1e3, 3)}
                if not ok:
                    pt["eligible"] = False
                points.append(pt)
                if log:
                    log(f"{ms:9.3f} ms  {opts}" + ("" if ok else "  (constraint not met)"))
        return cache[key]

    overall, overall_ms = None, float("inf")
    for sd in seeds:
        cur = dict(sd)
        for k in space:
            cur.setdefault(k, DEFAULT.get(k, space[k][0]))
        best = measure(cur)
        for _ in range(passes):
            start = best
            for k, values in space.items():
                for v in values:
                    if time.perf_counter() - t_start > budget_s:
                        break
                    cand = dict(cur)
                    cand[k] = v
                    ms = measure(cand)
                    if ms < best:
                        best, cur = ms, cand
            if best > 0.99 * start:
                break
        if best < overall_ms:
            overall, overall_ms = cur, best
    if overall is None or overall_ms == float("inf"):
        raise RuntimeError("no point met the constraint")
    return {
        "best": overall,
        "ms": round(overall_ms, 4),
        "msamples_s": round(n_threads / overall_ms / 1e3, 3),
        "points": points,
    }


def load() -> Dict:
    return json.loads(TUNING_FILE.read_text()) if TUNING_FILE.exists() else {}


def tuned(kernel: str, workload: str = "default") -> Optional[Dict]:
    """The options stored for (kernel, workload), falling back to the
    kernel's default entry; None when the kernel was never tuned."""
    t = load().get(kernel, {})
    e = t.get(workload) or t.get("default")
    return None if e is None else dict(e["best"])


def store(kernel: str, workload: str, result: Dict, device: str = "", keep_points: int = 12) -> None:
    data = load()
    entry = {
        "best": result["best"],
        "ms": result["ms"],
        "msamples_s": result["msamples_s"],
        "device": device,
        "points": sorted(result["points"], key=lambda p: (not p.get("eligible", True), p["ms"]))[:keep_points],
    }
    data.setdefault(kernel, {})[workload] = entry
    TUNING_FILE.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")
