"""Benchmark: Loom kernels on one B200, regrouped vs plain.

Workload (default): the Collatz stopping-time kernel on 2^24 threads,
n uniform in [1, 2^32) from SplitMix64 (seed 1), u64 arithmetic, u32 output.
A step is one launch of the regrouping engine over all 2^24 threads with the
inputs resident in HBM (128 MiB in + 64 MiB out per step, larger than the
126 MB L2, so no flush is needed between steps).  `value` is Loom threads
completed per second (Msamples/s) of the regrouping engine; the plain engine
is timed the same way beside it.  `e2e` is the same metric through the
public API with pinned host buffers (H2D of the inputs and D2H of the outputs
inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload collatz|fib]

Under torchrun each rank runs the full workload on its own GPU (weak
scaling, no data-path collective; Loom threads are independent), times with
CUDA events and reports the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

WORKLOADS = {
    "collatz": dict(
        kernel="collatz_u64",
        n=1 << 24,
        desc="Collatz stopping time, 2^24 threads, n ~ U[1, 2^32) (SplitMix64 seed 1), u64 -> steps:u32",
        lo=1,
        hi=(1 << 32) - 1,
        in_bytes=8,
        out_bytes=4,
        dtype="u64",
    ),
    "fib": dict(
        kernel="fib_u64",
        n=1 << 20,
        desc="Fibonacci (Loom README IR), 2^20 threads, n ~ U{0..93} (SplitMix64 seed 1), u64",
        lo=0,
        hi=93,
        in_bytes=8,
        out_bytes=8,
        dtype="u64",
    ),
}


def make_inputs(w):
    from oracle import oracle as O

    return O.uniform_int(1, w["n"], w["lo"], w["hi"])


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = ROOT / "gpurun_out" / f"clocks_rank{index}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                [
                    "nvidia-smi",
                    f"--id={self.index}",
                    f"--query-gpu={self.FIELDS}",
                    "--format=csv,noheader,nounits",
                    "-lms",
                    "200",
                ],
                stdout=self.f,
                stderr=subprocess.DEVNULL,
            )
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.path.read_text().splitlines():
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": smax,
            "samples": len(sm),
            "reasons": sorted(reasons),
        }


# ---------------------------------------------------------------- CPU arm
def cpu_reference(w, x, target_s: float = 4.0):
    """Loom's bse (oracle/_ref) on all host cores over a bounded sample;
    falls back to the C restatement (single thread) where bse was not
    built.  Returns (Msamples/s, info)."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    name = w["kernel"]
    if O.ref_available():
        kind = "reference"

        def run(m):
            O.ref_run(name, [x[:m]], m, threads=cores)

        used = cores
    else:
        kind = "port"
        it = O.Interp(name)

        def run(m):
            it.run([x[:m]])

        used = 1
    m = 1 << 14
    while True:
        t0 = time.perf_counter()
        run(m)
        dt = time.perf_counter() - t0
        if dt > target_s / 8 or m >= len(x):
            break
        m = min(len(x), m * 4)
    m = min(len(x), max(m, int(m * target_s / max(dt, 1e-9))))
    t0 = time.perf_counter()
    run(m)
    dt = time.perf_counter() - t0
    cpu = _cpu_model()
    return m / dt / 1e6, {
        "unit": "Msamples/s",
        "cores": used,
        "kind": kind,
        "sample": f"first {m} threads of the workload ({cpu}; {'Loom bse, g++ -O2 -mfma, std::thread per core' if kind == 'reference' else 'C restatement of bse, 1 thread'})",
        "seconds": round(dt, 3),
    }


def _cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown CPU"


# ---------------------------------------------------------------- GPU arm
def time_steps(fn, steps: int, warmup: int, torch, dist=None):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(steps):
        fn()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    torch.cuda.synchronize()
    return ms


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="collatz", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    config = {
        "workload": w["desc"],
        "kernel": w["kernel"],
        "threads_per_gpu": w["n"],
        "l2": "inputs larger than L2 (no flush)" if w["n"] * w["in_bytes"] > 126e6 else "L2 flushed between steps",
        "parallelism": f"replicas{world}" if world > 1 else "single",
    }

    if args.impl == "reference":
        if rank != 0:
            return
        x = make_inputs(w)
        vals = []
        info = None
        for i in range(warmup + args.steps):
            v, info = cpu_reference(w, x, target_s=2.0)
            if i >= warmup:
                vals.append(v)
        value = statistics.median(vals)
        print(
            json.dumps(
                {
                    "impl": "reference",
                    "metric": "Msamples/s (Loom threads completed per second)",
                    "value": round(value, 3),
                    "unit": "Msamples/s",
                    "n_gpus": args.gpus,
                    "steps": args.steps,
                    "warmup": warmup,
                    "higher_is_better": True,
                    "scaling": "weak",
                    "vs_baseline": None,
                    "dtype": w["dtype"],
                    "data": "synthetic",
                    "config": config,
                    "cpu_baseline": dict(info, value=round(value, 3)),
                    "e2e": {"value": round(value, 3), "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                }
            )
        )
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod
    else:
        torch.cuda.set_device(0)

    from loom_b200 import api

    n = w["n"]
    x = make_inputs(w)
    d_in = torch.from_numpy(x.view(np.int64)).cuda()
    out_dt = torch.int32 if w["out_bytes"] == 4 else torch.int64
    d_out = torch.empty(n, dtype=out_dt, device="cuda")
    # a dedicated stream: the library launches on it and the CUDA events of
    # time_steps are recorded on it (torch's current stream)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    res = {}
    for mode in ("plain", "regroup"):
        f = api.Function(w["kernel"], 0, mode)
        step = lambda: f.run_device([d_in], [d_out], n, stream=stream)  # noqa: E731
        ms = time_steps(step, args.steps, warmup, torch, dist)
        f.sync()
        f.reset_stats()
        # one counted launch for lane efficiency (plain needs its profiling variant)
        if mode == "plain":
            f.set_opts("plain", profile=True)
        f.run_device([d_in], [d_out], n, stream=stream)
        torch.cuda.synchronize()
        st = f.stats(raise_on_device_error=True)
        res[mode] = dict(ms=ms, stats=st, fn=f)

    # clocks: sample during a second timed pass of the headline engine
    f = res["regroup"]["fn"]
    f.set_opts("regroup")
    f.reset_stats()
    with ClockSampler(local) as clk:
        ms_r = time_steps(lambda: f.run_device([d_in], [d_out], n, stream=stream), args.steps, warmup, torch, dist)
    st_r = f.stats(raise_on_device_error=True)
    kern_ms = st_r["ms"]  # last launch, device time of the megakernel stream span

    # parity of this run
    got = d_out.cpu().numpy().view(np.uint32 if w["out_bytes"] == 4 else np.uint64)
    from oracle import oracle as O

    idx = O.uniform_int(5, 4096, 0, n - 1).astype(np.int64)
    (want,) = O.Interp(w["kernel"]).run([x[idx]])
    parity_ok = bool(np.array_equal(got[idx], want))

    # e2e through the public API with pinned host buffers
    h_in = torch.from_numpy(x.view(np.int64)).pin_memory()
    h_out = torch.empty(n, dtype=out_dt).pin_memory()
    fe = api.Function(w["kernel"], n, "regroup")
    e2e_step = lambda: fe.run_host_ptrs([h_in], [h_out], n)  # noqa: E731
    for _ in range(warmup):
        e2e_step()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_ok = bool(np.array_equal(h_out.numpy().view(got.dtype)[idx], want))

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    ms_step = ms_r / args.steps
    value = world * n / (ms_step / 1e3) / 1e6
    plain_ms = res["plain"]["ms"] / args.steps
    plain_value = world * n / (plain_ms / 1e3) / 1e6
    sr = res["regroup"]["stats"]
    sp = res["plain"]["stats"]
    # algorithmic bytes of one megakernel launch: inputs + outputs + state file
    algo_bytes = n * (w["in_bytes"] + w["out_bytes"]) + sr["state_bytes"] / max(1, sr["launches"])
    achieved = algo_bytes / (kern_ms / 1e3) / 1e9

    cpu = None
    if not args.no_cpu:
        v, info = cpu_reference(w, x)
        cpu = dict(info, value=round(v, 3))

    line = {
        "metric": "Msamples/s (Loom threads completed per second), regrouped engine; plain engine and SIMT lane efficiency beside it",
        "value": round(value, 3),
        "unit": "Msamples/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": warmup,
        "ms_per_step": round(ms_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": w["dtype"],
        "data": "synthetic",
        "config": config,
        "plain": {
            "value": round(plain_value, 3),
            "ms_per_step": round(plain_ms, 4),
            "lane_efficiency": round(sp["lane_efficiency"], 4),
            "kernel_ms_profiled": round(sp["ms"], 4),
        },
        "regroup": {
            "kernel_ms": round(kern_ms, 4),
            "lane_efficiency": round(sr["lane_efficiency"], 4),
            "rounds": sr["rounds"],
            "parks_per_thread": round(sr["parks"] / n, 4),
            "state_bytes_per_launch": int(sr["state_bytes"]),
        },
        "speedup_regroup_vs_plain": round(plain_ms / ms_step, 4),
        "parity": {"sample_threads": len(idx), "device_ok": parity_ok, "e2e_ok": e2e_ok},
        "roofline": {
            "bound": "hbm",
            "achieved": round(achieved, 2),
            "peak": hbm_peak,
            "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 5),
            "traffic": None,
            "peak_source": peak_src,
            "note": "algorithmic bytes = inputs + outputs + state-file saves/restores; the engines are SIMT-issue-bound, see profiles/",
        },
        "cpu_baseline": cpu,
        "e2e": {
            "value": round(world * n * args.steps / e2e_s / 1e6, 3),
            "unit": "Msamples/s",
            "h2d_bytes_per_step": n * w["in_bytes"],
            "d2h_bytes_per_step": n * w["out_bytes"],
        },
        "gpu_launches": 2 * args.steps,
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    for r in res.values():
        r["fn"].close()
    fe.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
