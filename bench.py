"""Benchmark: Loom kernels on one B200, regrouped vs plain.

Default workload (`--workload pt`): the FP32 sphere path tracer
(loom_b200/kernels/sphere_pt.hpp) rendering the Cornell box of spheres at
1024x768 with 64 samples per pixel: 50,331,648 Loom threads, one per
pixel-sample.  A step is one launch of the regrouping engine over all of
them.  The per-thread inputs (instance, sample index) are generated on the
device (no input traffic); the scene is a 304-byte table; the outputs are
three f32 columns (604 MB per step, larger than the 126 MB L2, so no flush
is needed between steps).  `value` is Loom threads completed per second
(Msamples/s) of the regrouping engine; the plain engine is timed the same
way beside it.  `e2e` is the same metric through the public API with host
buffers: the table copied in and the three output columns copied back to
pinned host memory inside the timed region.

Other workloads: `--workload collatz` (2^24 threads, n ~ U[1, 2^32)),
`--workload fib` (2^20 threads, n ~ U{0..93}).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload pt|collatz|fib]

Under torchrun each rank runs the full workload on its own GPU (weak
scaling, no data-path collective: Loom threads are independent), times with
CUDA events and reports the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

# Regrouping options per workload, from the sweeps kept in profiles/
TUNED = {
    "sphere_pt_f32": dict(burst=4, utr_lanes=8, population=1 << 21, block_size=256, period=4096),
    "collatz_u64": dict(burst=64, utr_lanes=16, block_size=512, period=65536, prefetch=False),
    "fib_u64": dict(burst=64, utr_lanes=16, block_size=512, period=1024, prefetch=False),
}


# ---------------------------------------------------------------- workloads
class Workload:
    kernel = ""
    desc = ""
    dtype = ""

    def prepare(self, torch, device: bool = True):
        raise NotImplementedError


class PathTracing(Workload):
    kernel = "sphere_pt_f32"
    dtype = "f32"

    def __init__(self, width=1024, height=768, spp=64):
        from loom_b200 import scenes as S

        self.S = S
        self.req = S.cornell_request(width, height, spp, seed=1)
        self.table, self.starts = S.pack([self.req])
        self.n = self.req.threads
        self.desc = (
            f"sphere path tracer, Cornell box of 9 spheres (walls r=1e5, mirror, glass IOR 1.5, light), "
            f"{width}x{height} x {spp} spp = {self.n} threads, FP32, RR from depth 5, max depth 16"
        )
        self.in_bytes = 0
        self.out_bytes = 12

    def inputs(self, api):
        return [api.Broadcast(0, "u32"), api.Iota()]

    def device_buffers(self, torch):
        self.d_table = torch.from_numpy(self.table.view(np.int32)).cuda()
        self.d_out = [torch.empty(self.n, dtype=torch.float32, device="cuda") for _ in range(3)]

    def launch(self, f, api, stream):
        f.launch_device(self.inputs(api), self.d_out, self.n, table=self.d_table, stream=stream)

    def check(self, api):
        """Bit-exact parity of a seeded sample against the C oracle."""
        from oracle import oracle as O

        got = [o.cpu().numpy() for o in self.d_out]
        idx = np.sort(O.uniform_int(5, 256, 0, self.n - 1).astype(np.int64))
        ins = O.expand_inputs(["instance", "local_iota"], self.n, self.starts, ["u32", "u32"])
        want = O.Interp(self.kernel).run([a[idx] for a in ins], table=self.table)
        return all(np.array_equal(g[idx].view(np.uint32), w.view(np.uint32)) for g, w in zip(got, want)), idx

    def e2e(self, api, torch, steps, warmup, dist):
        h_out = [torch.empty(self.n, dtype=torch.float32).pin_memory() for _ in range(3)]
        fe = api.Function(self.kernel, self.n, "regroup", **TUNED[self.kernel])

        def step():
            L, keep = fe._launch_struct(self.inputs(api), h_out, self.n, None, self.table)
            api.check(api.lib().loom_b200_launch_host(fe._h, api.ctypes.byref(L)))

        for _ in range(warmup):
            step()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        dt = time.perf_counter() - t0
        got = [h.numpy() for h in h_out]
        ok = all(np.array_equal(g, d.cpu().numpy()) for g, d in zip(got, self.d_out))
        fe.close()
        return dt, ok, self.table.nbytes, 3 * 4 * self.n

    def cpu_inputs(self):
        from oracle import oracle as O

        return O.expand_inputs(["instance", "local_iota"], self.n, self.starts, ["u32", "u32"]), self.table


class IntegerLoop(Workload):
    def __init__(self, kernel, n, lo, hi, out_bytes, desc):
        self.kernel = kernel
        self.n = n
        self.lo, self.hi = lo, hi
        self.desc = desc
        self.dtype = "u64"
        self.in_bytes = 8
        self.out_bytes = out_bytes
        from oracle import oracle as O

        self.x = O.uniform_int(1, n, lo, hi)

    def device_buffers(self, torch):
        self.d_in = torch.from_numpy(self.x.view(np.int64)).cuda()
        dt = torch.int32 if self.out_bytes == 4 else torch.int64
        self.d_out = torch.empty(self.n, dtype=dt, device="cuda")

    def launch(self, f, api, stream):
        f.run_device([self.d_in], [self.d_out], self.n, stream=stream)

    def check(self, api):
        from oracle import oracle as O

        got = self.d_out.cpu().numpy().view(np.uint32 if self.out_bytes == 4 else np.uint64)
        idx = O.uniform_int(5, 4096, 0, self.n - 1).astype(np.int64)
        (want,) = O.Interp(self.kernel).run([self.x[idx]])
        return bool(np.array_equal(got[idx], want)), idx

    def e2e(self, api, torch, steps, warmup, dist):
        h_in = torch.from_numpy(self.x.view(np.int64)).pin_memory()
        h_out = torch.empty(self.n, dtype=self.d_out.dtype).pin_memory()
        fe = api.Function(self.kernel, self.n, "regroup", **TUNED[self.kernel])
        for _ in range(warmup):
            fe.run_host_ptrs([h_in], [h_out], self.n)
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            fe.run_host_ptrs([h_in], [h_out], self.n)
        dt = time.perf_counter() - t0
        ok = bool(np.array_equal(h_out.numpy(), self.d_out.cpu().numpy()))
        fe.close()
        return dt, ok, self.n * self.in_bytes, self.n * self.out_bytes

    def cpu_inputs(self):
        return [self.x], None


def make_workload(name):
    if name == "pt":
        return PathTracing()
    if name == "pt_small":  # the profiling case: same scene at 256x192
        return PathTracing(256, 192, 64)
    if name == "collatz":
        return IntegerLoop(
            "collatz_u64", 1 << 24, 1, (1 << 32) - 1, 4,
            "Collatz stopping time, 2^24 threads, n ~ U[1, 2^32) (SplitMix64 seed 1), u64 -> steps:u32",
        )
    if name == "fib":
        return IntegerLoop(
            "fib_u64", 1 << 20, 0, 93, 8,
            "Fibonacci (Loom README IR), 2^20 threads, n ~ U{0..93} (SplitMix64 seed 1), u64",
        )
    raise ValueError(name)


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
def cpu_reference(w, target_s: float = 4.0):
    """Loom's bse (oracle/_ref) on all host cores over a bounded sample of
    the workload's threads; falls back to the C restatement (one thread)
    where bse was not built.  Returns (Msamples/s, info)."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    ins, table = w.cpu_inputs()
    # a seeded random subset of the workload's threads (cost per thread
    # varies across the image; a prefix would not be representative)
    perm = np.random.default_rng(7).permutation(w.n)
    ins = [np.ascontiguousarray(a[perm]) for a in ins]
    if O.ref_available():
        kind = "reference"

        def run(m):
            O.ref_run(w.kernel, [a[:m] for a in ins], m, threads=cores, table=table)

        used = cores
    else:
        kind = "port"
        it = O.Interp(w.kernel)

        def run(m):
            it.run([a[:m] for a in ins], table=table)

        used = 1
    m = 1 << 12
    while True:
        t0 = time.perf_counter()
        run(m)
        dt = time.perf_counter() - t0
        if dt > target_s / 8 or m >= w.n:
            break
        m = min(w.n, m * 4)
    m = min(w.n, max(m, int(m * target_s / max(dt, 1e-9))))
    t0 = time.perf_counter()
    run(m)
    dt = time.perf_counter() - t0
    cpu = _cpu_model()
    how = (
        "Loom bse (vm::bse::function), g++ -O2 -mfma, one std::thread per core"
        if kind == "reference"
        else "C restatement of bse, one thread"
    )
    return m / dt / 1e6, {
        "unit": "Msamples/s",
        "cores": used,
        "kind": kind,
        "sample": f"{m} threads drawn at random (seed 7) from the workload's {w.n}, on {cpu}; {how}",
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
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="pt", choices=["pt", "pt_small", "collatz", "fib"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    w = make_workload(args.workload)
    config = {
        "workload": w.desc,
        "kernel": w.kernel,
        "threads_per_gpu": w.n,
        "l2": "outputs larger than L2 (no flush)",
        "parallelism": f"replicas{world}" if world > 1 else "single",
        "regroup_options": TUNED[w.kernel],
    }
    metric = "Msamples/s (Loom threads completed per second), regrouped engine; plain engine and SIMT lane efficiency beside it"

    if args.impl == "reference":
        if rank != 0:
            return
        vals, info = [], None
        for i in range(warmup + args.steps):
            v, info = cpu_reference(w, target_s=2.0)
            if i >= warmup:
                vals.append(v)
        value = statistics.median(vals)
        print(
            json.dumps(
                {
                    "impl": "reference",
                    "metric": metric,
                    "value": round(value, 3),
                    "unit": "Msamples/s",
                    "n_gpus": args.gpus,
                    "steps": args.steps,
                    "warmup": warmup,
                    "higher_is_better": True,
                    "scaling": "weak",
                    "vs_baseline": None,
                    "dtype": w.dtype,
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

    # a dedicated stream: the library launches on it and the CUDA events of
    # time_steps are recorded on it (torch's current stream)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    w.device_buffers(torch)

    res = {}
    for mode in ("plain", "regroup"):
        opts = TUNED[w.kernel] if mode == "regroup" else {}
        f = api.Function(w.kernel, 0, mode, **opts)
        ms = time_steps(lambda: w.launch(f, api, stream), args.steps, warmup, torch, dist)
        f.sync()
        f.reset_stats()
        f.set_opts(mode, profile=True, **opts)  # one counted launch for lane efficiency
        w.launch(f, api, stream)
        torch.cuda.synchronize()
        st = f.stats(raise_on_device_error=True)
        f.set_opts(mode, **opts)
        f.reset_stats()
        res[mode] = dict(ms=ms, stats=st, fn=f)
    plain_out_ok, _ = w.check(api)

    # the headline: the regrouping engine, clocks sampled during the timed region
    f = res["regroup"]["fn"]
    with ClockSampler(local) as clk:
        ms_r = time_steps(lambda: w.launch(f, api, stream), args.steps, warmup, torch, dist)
    st_r = f.stats(raise_on_device_error=True)
    kern_ms = st_r["ms"]
    parity_ok, idx = w.check(api)

    e2e_s, e2e_ok, h2d, d2h = w.e2e(api, torch, args.steps, warmup, dist)
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

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
    value = world * w.n / (ms_step / 1e3) / 1e6
    plain_ms = res["plain"]["ms"] / args.steps
    plain_value = world * w.n / (plain_ms / 1e3) / 1e6
    sr = res["regroup"]["stats"]
    sp = res["plain"]["stats"]
    # algorithmic bytes of one megakernel launch: inputs, outputs, table and
    # the queue state the engine moved (saves + restores, counted in-kernel)
    state_per_launch = st_r["state_bytes"] / max(1, st_r["launches"])
    algo_bytes = w.n * (w.in_bytes + w.out_bytes) + state_per_launch
    achieved = algo_bytes / (kern_ms / 1e3) / 1e9

    # DRAM traffic of the dominant kernel from an ncu capture (per thread,
    # scaled to this launch), see profiles/roofline_traffic.json
    traffic = None
    tf = ROOT / "profiles" / "roofline_traffic.json"
    if tf.exists():
        t = json.loads(tf.read_text()).get(w.kernel)
        if t:
            traffic = int(t["dram_bytes_per_thread"] * w.n)

    cpu = None
    if not args.no_cpu:
        v, info = cpu_reference(w)
        cpu = dict(info, value=round(v, 3))

    line = {
        "metric": metric,
        "value": round(value, 3),
        "unit": "Msamples/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": warmup,
        "ms_per_step": round(ms_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": w.dtype,
        "data": "synthetic",
        "config": config,
        "plain": {
            "value": round(plain_value, 3),
            "ms_per_step": round(plain_ms, 4),
            "lane_efficiency": round(sp["lane_efficiency"], 4),
        },
        "regroup": {
            "kernel_ms": round(kern_ms, 4),
            "lane_efficiency": round(sr["lane_efficiency"], 4),
            "rounds": int(st_r["rounds"] / max(1, st_r["launches"])),
            "parks_per_thread": round(st_r["parks"] / max(1, st_r["launches"]) / w.n, 4),
            "state_bytes_per_launch": int(state_per_launch),
        },
        "speedup_regroup_vs_plain": round(plain_ms / ms_step, 4),
        "lane_efficiency_note": "VM instructions executed / (32 x VM instructions issued per warp), in-kernel counters of a profiled launch",
        "parity": {
            "sample_threads": int(len(idx)),
            "regroup_device_ok": bool(parity_ok),
            "plain_device_ok": bool(plain_out_ok),
            "e2e_ok": bool(e2e_ok),
        },
        "roofline": {
            "bound": "hbm",
            "achieved": round(achieved, 2),
            "peak": hbm_peak,
            "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 5),
            "traffic": traffic,
            "algorithmic_bytes": int(algo_bytes),
            "peak_source": peak_src,
            "note": "algorithmic bytes = outputs + inputs + queue-state saves/restores of the regrouping megakernel; the engine is SIMT issue/latency bound, not HBM bound (profiles/)",
        },
        "cpu_baseline": cpu,
        "e2e": {
            "value": round(world * w.n * args.steps / e2e_s / 1e6, 3),
            "unit": "Msamples/s",
            "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h),
        },
        "gpu_launches": 2 * args.steps,
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    for r in res.values():
        r["fn"].close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
