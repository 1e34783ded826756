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

Other workloads:
  batch    256 render requests of uneven size, each with its own random
           scene, in one launch (392.8 M threads)
  collatz  2^24 threads, n ~ U[1, 2^32)
  fib      2^20 threads, n ~ U{0..93}
  loom_pt, loom_pt2
           Loom's own path tracers (pt_const, pt2_const) at the 40x40
           configurations of its published CPU results
  loom_pt_512, loom_pt2_512
           the same programs at 512x512 pixels (262,144 threads)
  loom_primary, loom_primary_b20
           Loom's primary-ray tracer (primary_const) at its benchmark's
           configuration: 256x256 pixels, 64 samples, blur 1 or 20
  serve    the serving loop: Poisson arrivals of a request mix (60 % render
           requests as in `batch`, 20 % Collatz batches of 2^16-2^22 inputs,
           20 % Fibonacci batches of 2^16-2^20 inputs) at 25/50/75/100 % of
           the measured capacity; throughput and p50/p99 latency of the
           continuous-batching servers beside a plain-engine FIFO queue.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload pt|pt_small|batch|collatz|fib|loom_pt|loom_pt2|loom_pt_512|loom_pt2_512|
                                loom_primary|loom_primary_b20|serve]

Under torchrun each rank runs the full workload on its own GPU (weak
scaling, no data-path collective: Loom threads are independent), times with
CUDA events and reports the max over ranks.

The CPU leg (skipped with --no-cpu) times Loom's own scalar backend on the
host cores and is also the parity check: the reference's outputs for a
seeded sample of threads are compared bit for bit with both engines'.
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

# Regrouping options: the autotuner's results (loom_b200/tuning.json, made
# by `bench.py --tune`), per kernel and workload; these are the seeds used
# where a kernel was never tuned.
FALLBACK = {
    "sphere_pt_f32": dict(burst=4, utr_lanes=8, population=1 << 21, block_size=256, period=4096),
    "collatz_u64": dict(burst=64, utr_lanes=16, block_size=512, period=65536, prefetch=False),
    "fib_u64": dict(burst=64, utr_lanes=16, block_size=512, period=1024, prefetch=False),
    "pt_const_40": dict(cost_model=True, utr_lanes=4, burst=32, block_size=128),
    "pt2_const_40": dict(cost_model=True, utr_lanes=4, burst=32, block_size=128),
    # Loom's own path tracers: per-block stepping in reverse post-order was
    # the fastest regrouping form measured (the plain engine is faster still)
    "pt_const_512": dict(schedule=2, burst=64, period=1 << 20, prefetch=False, utr_lanes=1),
    "pt2_const_512": dict(schedule=2, burst=64, period=1 << 20, prefetch=False, utr_lanes=1),
    "primary_const_256": dict(schedule=2, burst=64, period=1 << 20, prefetch=False, utr_lanes=1),
    "primary_const_b20_256": dict(schedule=2, burst=64, period=1 << 20, prefetch=False, utr_lanes=1),
}


def regroup_opts(kernel: str, key: str = "default") -> dict:
    from loom_b200 import autotune as T

    t = T.tuned(kernel, key)
    return dict(t) if t else dict(FALLBACK[kernel])


CHECK_THREADS = 1 << 14  # threads compared with the reference


# ---------------------------------------------------------------- workloads
class Workload:
    kernel = ""
    tune_key = "default"
    desc = ""
    dtype = ""
    n = 0
    in_bytes = 0
    out_bytes = 0

    def check_tids(self) -> np.ndarray:
        """A seeded sample of thread ids for the parity check."""
        rng = np.random.default_rng(5)
        return np.unique(rng.integers(0, self.n, size=min(CHECK_THREADS, self.n)))

    def outputs_at(self, tids):
        """Device outputs of threads `tids` (host arrays, one per output)."""
        import torch

        ix = torch.from_numpy(np.ascontiguousarray(tids, dtype=np.int64)).cuda()
        return [o[ix].cpu().numpy() for o in self.d_out]


class PathTracing(Workload):
    kernel = "sphere_pt_f32"
    dtype = "f32"
    tune_key = "pt"

    def __init__(self, width=1024, height=768, spp=64):
        from loom_b200 import scenes as S

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

    def ref_inputs(self, tids):
        tids = np.asarray(tids, dtype=np.uint64)
        return [np.zeros(len(tids), dtype=np.uint32), tids.astype(np.uint32)], self.table

    def e2e(self, api, torch, steps, warmup, dist):
        h_out = [torch.empty(self.n, dtype=torch.float32).pin_memory() for _ in range(3)]
        fe = api.Function(self.kernel, self.n, "regroup", **self.opts)

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
        ok = all(torch.equal(h, d.cpu()) for h, d in zip(h_out, self.d_out))
        fe.close()
        return dt, ok, self.table.nbytes, 3 * 4 * self.n


class BatchedPathTracing(PathTracing):
    """Many render requests of uneven size in one launch: each request has
    its own resolution, sample count and random scene (loom_b200.scenes
    .random_request); threads of all requests share the megakernel and are
    mapped to (request, sample) on the device from the instance offsets."""

    tune_key = "batch"

    def __init__(self, count=256, seed=3):
        from loom_b200 import scenes as S

        rng = np.random.default_rng(seed)
        self.reqs = [S.random_request(rng, seed=i + 1) for i in range(count)]
        self.table, self.starts = S.pack(self.reqs)
        self.n = int(self.starts[-1])
        self.desc = (
            f"{count} batched render requests (seed {seed}): resolution from {{64,128,256,512}}^2, spp from "
            f"{{1,4,16,64}}, 8-64 random spheres each (60/20/20 diffuse/mirror/glass, 1-4 emitters), "
            f"{self.n} threads in one launch, FP32"
        )
        self.in_bytes = 0
        self.out_bytes = 12

    def inputs(self, api):
        return [api.Instance(), api.LocalIota()]

    def device_buffers(self, torch):
        super().device_buffers(torch)
        self.d_starts = torch.from_numpy(self.starts.view(np.int64)).cuda()

    def launch(self, f, api, stream):
        f.launch_device(
            self.inputs(api), self.d_out, self.n, instance_starts=self.d_starts, table=self.d_table, stream=stream
        )

    def check_tids(self):
        """4 random threads of every request."""
        rng = np.random.default_rng(5)
        lo, hi = self.starts[:-1].astype(np.int64), self.starts[1:].astype(np.int64)
        return np.unique(np.concatenate([rng.integers(a, b, size=4) for a, b in zip(lo, hi)]))

    def ref_inputs(self, tids):
        tids = np.asarray(tids, dtype=np.uint64)
        inst = (np.searchsorted(self.starts, tids, side="right") - 1).astype(np.int64)
        return [inst.astype(np.uint32), (tids - self.starts[inst]).astype(np.uint32)], self.table

    def e2e(self, api, torch, steps, warmup, dist):
        h_out = [torch.empty(self.n, dtype=torch.float32).pin_memory() for _ in range(3)]
        fe = api.Function(self.kernel, self.n, "regroup", **self.opts)

        def step():
            L, keep = fe._launch_struct(self.inputs(api), h_out, self.n, self.starts, self.table)
            api.check(api.lib().loom_b200_launch_host(fe._h, api.ctypes.byref(L)))

        for _ in range(warmup):
            step()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        dt = time.perf_counter() - t0
        ok = all(torch.equal(h, d.cpu()) for h, d in zip(h_out, self.d_out))
        fe.close()
        return dt, ok, self.table.nbytes + self.starts.nbytes, 3 * 4 * self.n


class IntegerLoop(Workload):
    def __init__(self, kernel, n, lo, hi, out_bytes, desc):
        from loom_b200 import inputs as I

        self.kernel = kernel
        self.n = n
        self.desc = desc
        self.dtype = "u64"
        self.in_bytes = 8
        self.out_bytes = out_bytes
        self.x = I.uniform_int(1, n, lo, hi)

    def device_buffers(self, torch):
        self.d_in = torch.from_numpy(self.x.view(np.int64)).cuda()
        dt = torch.int32 if self.out_bytes == 4 else torch.int64
        self.d_out = [torch.empty(self.n, dtype=dt, device="cuda")]

    def launch(self, f, api, stream):
        f.run_device([self.d_in], self.d_out, self.n, stream=stream)

    def ref_inputs(self, tids):
        return [self.x[np.asarray(tids, dtype=np.int64)]], None

    def e2e(self, api, torch, steps, warmup, dist):
        h_in = torch.from_numpy(self.x.view(np.int64)).pin_memory()
        h_out = torch.empty(self.n, dtype=self.d_out[0].dtype).pin_memory()
        fe = api.Function(self.kernel, self.n, "regroup", **self.opts)
        for _ in range(warmup):
            fe.run_host_ptrs([h_in], [h_out], self.n)
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            fe.run_host_ptrs([h_in], [h_out], self.n)
        dt = time.perf_counter() - t0
        ok = bool(torch.equal(h_out, self.d_out[0].cpu()))
        fe.close()
        return dt, ok, self.n * self.in_bytes, self.n * self.out_bytes


class LoomPathTracer(Workload):
    """Loom's own path tracers (src/smallpt/vm/pt.hpp) at the 40x40
    configurations of its published results: one Loom thread per pixel,
    adaptive sampling up to 64 samples (blur 1, depth 2, threshold 1e-4 for
    pt_const, 1e-3 for pt2_const).  A step renders the image once."""

    dtype = "f32"

    def __init__(self, kernel, threshold, side=40, blur=1):
        self.kernel = kernel
        self.tune_key = "default"
        x, y = np.meshgrid(np.arange(side, dtype=np.uint32), np.arange(side, dtype=np.uint32))
        self.pixels = ((x << 16) | y).reshape(-1)
        self.n = len(self.pixels)
        if threshold is None:  # primary rays: a fixed sample count, no bounces
            self.desc = (
                f"Loom's primary_const (src/smallpt/vm/pt.hpp), {side}x{side} pixels, 64 primary-ray samples "
                f"per pixel, blur {blur}: one thread per pixel, {self.n} threads per step"
            )
        else:
            self.desc = (
                f"Loom's {kernel.rsplit('_', 1)[0]} (src/smallpt/vm/pt.hpp), {side}x{side} pixels, up to 64 adaptive "
                f"samples, blur {blur}, threshold {threshold}, depth 2: one thread per pixel, {self.n} threads per step"
            )
        self.in_bytes = 4
        self.out_bytes = 20

    def device_buffers(self, torch):
        self.d_in = torch.from_numpy(self.pixels.view(np.int32)).cuda()
        self.d_out = [torch.empty(self.n, dtype=torch.float32, device="cuda") for _ in range(3)]
        self.d_out += [torch.empty(self.n, dtype=torch.int32, device="cuda") for _ in range(2)]

    def launch(self, f, api, stream):
        f.run_device([self.d_in], self.d_out, self.n, stream=stream)

    def ref_inputs(self, tids):
        return [self.pixels[np.asarray(tids, dtype=np.int64)]], None

    def e2e(self, api, torch, steps, warmup, dist):
        h_in = torch.from_numpy(self.pixels.view(np.int32)).pin_memory()
        h_out = [torch.empty(self.n, dtype=o.dtype).pin_memory() for o in self.d_out]
        fe = api.Function(self.kernel, self.n, "regroup", **self.opts)
        for _ in range(warmup):
            fe.run_host_ptrs([h_in], h_out, self.n)
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            fe.run_host_ptrs([h_in], h_out, self.n)
        dt = time.perf_counter() - t0
        ok = all(torch.equal(h, d.cpu()) for h, d in zip(h_out, self.d_out))
        fe.close()
        return dt, ok, self.n * self.in_bytes, self.n * self.out_bytes


def make_workload(name):
    if name == "loom_pt":
        return LoomPathTracer("pt_const_40", "1e-4")
    if name == "loom_pt2":
        return LoomPathTracer("pt2_const_40", "1e-3")
    if name == "loom_pt_512":
        return LoomPathTracer("pt_const_512", "1e-4", 512)
    if name == "loom_pt2_512":
        return LoomPathTracer("pt2_const_512", "1e-3", 512)
    if name == "loom_primary":
        return LoomPathTracer("primary_const_256", None, 256)
    if name == "loom_primary_b20":
        return LoomPathTracer("primary_const_b20_256", None, 256, blur=20)
    if name == "pt":
        return PathTracing()
    if name == "pt_small":  # the profiling case: same scene at 256x192
        return PathTracing(256, 192, 64)
    if name == "batch":
        return BatchedPathTracing()
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
        # LOOM_B200_CLOCKS_DIR keeps the raw samples; by default they go to a
        # temporary directory and only the summary reaches the bench line
        import tempfile

        d = os.environ.get("LOOM_B200_CLOCKS_DIR") or tempfile.mkdtemp(prefix="loom_b200_clocks_")
        self.path = pathlib.Path(d) / f"clocks_rank{index}.csv"

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
                    "50",
                ],
                stdout=self.f,
                stderr=subprocess.DEVNULL,
            )
            # the timed region starts once the first sample is in (nvidia-smi
            # takes a moment to come up), at most two seconds from now
            t_end = time.monotonic() + 2.0
            while time.monotonic() < t_end and self.proc.poll() is None:
                if self.path.stat().st_size > 0:
                    break
                time.sleep(0.02)
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


# ---------------------------------------------------------------- CPU leg
def _cpu_model() -> str:
    """CPU model and widest x86 vector ISA of the host (Loom reports both
    beside its CPU timings: src/benchmarks/bm.hpp:39-69, simd.hpp:66-77)."""
    model, flags = "unknown CPU", set()
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name") and model == "unknown CPU":
                model = ln.split(":", 1)[1].strip()
            elif ln.startswith("flags") and not flags:
                flags = set(ln.split(":", 1)[1].split())
    except Exception:
        pass
    isa = next((name for flag, name in (("avx512f", "AVX-512"), ("avx2", "AVX2"), ("avx", "AVX")) if flag in flags), "")
    return f"{model} ({isa})" if isa else model


def _reference_runner():
    """Loom's bse (oracle/_ref) on all host cores, else the C restatement on
    one core: returns (run(kernel, inputs, table) -> outputs, kind, cores)."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    if O.ref_available():

        def run(kernel, ins, table):
            return O.ref_run(kernel, ins, len(ins[0]), threads=cores, table=table)

        return run, "reference", cores

    def run(kernel, ins, table):
        return O.Interp(kernel).run(ins, table=table)

    return run, "port", 1


def cpu_reference(w, check_tids=None, target_s: float = 2.0):
    """Times the reference on a bounded random sample of the workload's
    threads (about `target_s` seconds of CPU work), and, with `check_tids`,
    returns the reference's outputs of those threads for the parity check.
    Returns (Msamples/s, info, outputs or None)."""
    run, kind, cores = _reference_runner()
    rng = np.random.default_rng(7)
    pool = rng.integers(0, w.n, size=min(w.n, 1 << 26))
    m = 1 << 12
    while True:
        ins, table = w.ref_inputs(pool[:m])
        t0 = time.perf_counter()
        run(w.kernel, ins, table)
        dt = time.perf_counter() - t0
        if dt > target_s / 8 or m >= len(pool):
            break
        m = min(len(pool), m * 4)
    m = min(len(pool), max(m, int(m * target_s / max(dt, 1e-9))))
    ins, table = w.ref_inputs(pool[:m])
    t0 = time.perf_counter()
    run(w.kernel, ins, table)
    dt = time.perf_counter() - t0
    how = (
        "Loom bse (vm::bse::function), g++ -O2 -mfma, one std::thread per core"
        if kind == "reference"
        else "C restatement of bse, one thread"
    )
    info = {
        "unit": "Msamples/s",
        "cores": cores,
        "kind": kind,
        "sample": f"{m} threads drawn at random (seed 7) from the workload's {w.n}, on {_cpu_model()}; {how}",
        "seconds": round(dt, 3),
    }
    want = None
    if check_tids is not None:
        ins, table = w.ref_inputs(check_tids)
        want = run(w.kernel, ins, table)
    return m / dt / 1e6, info, want


# Float outputs that pass through the host libm's sinf/cosf (Loom's
# pt2_const) are held within this many ulp of the reference; everything else
# is compared bit for bit.
ULP_TOLERANCE = {"pt2_const_40": 4, "pt2_const_512": 4}


def same_bits(got, want, kernel: str = "") -> bool:
    for g, w in zip(got, want):
        g, w = np.ascontiguousarray(g), np.ascontiguousarray(w)
        if kernel in ULP_TOLERANCE and w.dtype.kind == "f":
            ulps = np.abs(g.astype(np.float64) - w.astype(np.float64)) / np.spacing(np.abs(w)).astype(np.float64)
            if len(w) and float(ulps.max()) > ULP_TOLERANCE[kernel]:
                return False
        elif not np.array_equal(g.view(np.uint8), w.view(np.uint8)):
            return False
    return True


# ---------------------------------------------------------------- GPU arm
def ncu_rooflines(w, kern_ms: float, sm_mhz: float, path: pathlib.Path = None):
    """Figures of the dominant kernel that come from an ncu capture
    (profiles/roofline_traffic.json, per thread, scaled to this launch):
    DRAM traffic per launch, and the issue roofline — SASS warp instructions
    per second against one per cycle on each of the 148 x 4 SM
    sub-partitions at `sm_mhz`.  The issue figure is given only when the
    capture was taken with the same regrouping options.  Returns (traffic
    bytes or None, issue dict or None)."""
    tf = path or ROOT / "profiles" / "roofline_traffic.json"
    if not tf.exists():
        return None, None
    t = json.loads(tf.read_text()).get(w.tune_key)
    if not t or t.get("kernel") != w.kernel:
        return None, None
    traffic = int(t["dram_bytes_per_thread"] * w.n) if t.get("dram_bytes_per_thread") else None
    issue = None
    if t.get("sass_options") == w.opts and t.get("sass_warp_inst_per_thread") and kern_ms > 0:
        got = t["sass_warp_inst_per_thread"] * w.n / (kern_ms / 1e3) / 1e9
        top = 148 * 4 * sm_mhz / 1e3
        issue = {
            "achieved": round(got, 1),
            "peak": round(top, 1),
            "unit": "G warp instructions/s",
            "frac": round(got / top, 4),
            "sass_warp_inst_per_thread": t["sass_warp_inst_per_thread"],
        }
    return traffic, issue


def max_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    """The largest `x` over the ranks of the process group (every rank gets
    it); `x` itself without one.  NCCL groups reduce a CUDA tensor, gloo
    groups a CPU tensor."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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
        ms = max_over_ranks(ms, dist)
        dist.barrier()
    torch.cuda.synchronize()
    return ms


def base_line(args, warmup, world, w_desc, kernel, dtype, metric, extra=None):
    line = {
        "metric": metric,
        "unit": "Msamples/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": dtype,
        "data": "synthetic",
        "config": {
            "workload": w_desc,
            "kernel": kernel,
            "parallelism": f"replicas{world}" if world > 1 else "single",
        },
    }
    if extra:
        line["config"].update(extra)
    return line


METRIC = (
    "Msamples/s (Loom threads completed per second), regrouped engine; plain engine and SIMT lane "
    "efficiency beside it"
)

# Loom's benchmarks append one CSV row per run (date, repo hash, compiler,
# fast-math, CPU model, SIMD ISA, benchmark id, seconds;
# src/benchmarks/bm.hpp:103-139); `--csv PATH` appends the same kind of row,
# extended with the GPU figures of the bench line.
CSV_FIELDS = [
    "date", "repo_hash", "compiler", "device", "impl", "workload", "kernel", "n_gpus", "ms_per_step",
    "msamples_s", "plain_msamples_s", "lane_efficiency", "state_gbs", "issue_frac", "p50_ms", "p99_ms",
]


def csv_row(line: dict, device: str = "", compiler: str = "", repo_hash: str = "") -> dict:
    """The CSV row of a bench line (missing figures left empty)."""
    import datetime

    rg = line.get("regroup") or {}
    roof = line.get("roofline") or {}
    issue = line.get("issue_roofline") or {}
    cfg = line.get("config") or {}
    return {
        "date": datetime.datetime.now(datetime.timezone.utc).strftime("%Y-%m-%dT%H:%M:%SZ"),
        "repo_hash": repo_hash,
        "compiler": compiler,
        "device": device,
        "impl": line.get("impl", "b200"),
        "workload": cfg.get("workload", ""),
        "kernel": cfg.get("kernel", ""),
        "n_gpus": line.get("n_gpus", ""),
        "ms_per_step": line.get("ms_per_step", ""),
        "msamples_s": line.get("value", ""),
        "plain_msamples_s": (line.get("plain") or {}).get("value", ""),
        "lane_efficiency": rg.get("lane_efficiency", ""),
        "state_gbs": roof.get("achieved", ""),
        "issue_frac": issue.get("frac", ""),
        "p50_ms": line.get("p50_ms", ""),
        "p99_ms": line.get("p99_ms", ""),
    }


def append_csv(path: str, line: dict) -> None:
    """Appends the row of `line` to the CSV file at `path` (header first
    when the file is new)."""
    import csv
    import subprocess

    def out(cmd):
        try:
            return subprocess.run(cmd, capture_output=True, text=True, timeout=10, cwd=ROOT).stdout.strip()
        except Exception:
            return ""

    device = ""
    try:
        import torch

        if torch.cuda.is_available():
            device = torch.cuda.get_device_name(0)
    except Exception:
        pass
    nv = out(["nvcc", "--version"]).splitlines()
    row = csv_row(line, device, nv[-1] if nv else "", out(["git", "rev-parse", "--short", "HEAD"]))
    f = pathlib.Path(path)
    new = not f.exists() or f.stat().st_size == 0
    with open(f, "a", newline="") as fh:
        w = csv.DictWriter(fh, fieldnames=CSV_FIELDS)
        if new:
            w.writeheader()
        w.writerow(row)


# ---------------------------------------------------------------- serving
SERVE_KERNELS = {"pt": "sphere_pt_f32", "collatz": "collatz_u64", "fib": "fib_u64"}
SERVE_POOL = {"collatz": (1 << 23, 1, (1 << 32) - 1), "fib": (1 << 21, 0, 93)}
SERVE_BUDGET = 100 << 30  # device bytes for thread state, columns and tables


class ServeMix:
    """Seeded request stream: 60 % render requests drawn as in the batched
    workload, 20 % Collatz batches of 2^16-2^22 inputs, 20 % Fibonacci
    batches of 2^16-2^20 inputs (sizes log-uniform over the powers of two;
    inputs are slices of a seeded pool of each kind)."""

    def __init__(self, seed: int):
        self.rng = np.random.default_rng(seed)
        self.seed = seed
        self.k = 0

    def draw(self, count: int):
        from loom_b200 import scenes as S

        out = []
        for _ in range(count):
            self.k += 1
            u = self.rng.uniform()
            if u < 0.6:
                r = S.random_request(self.rng, seed=self.seed * 100003 + self.k)
                h, b = S.request_words(r)
                out.append(("pt", r.threads, dict(header=h, body=b), r))
            else:
                kind = "collatz" if u < 0.8 else "fib"
                lo, hi = (16, 22) if kind == "collatz" else (16, 20)
                n = 1 << int(self.rng.integers(lo, hi + 1))
                off = int(self.rng.integers(0, SERVE_POOL[kind][0] - n + 1))
                out.append((kind, n, off, None))
        return out


class PinnedPool:
    """Pinned host buffers by power-of-two size class, reused across
    requests (outputs of requests in flight)."""

    def __init__(self, torch):
        self.torch = torch
        self.free = {}

    def get(self, nbytes: int):
        c = 1 << max(12, math.ceil(math.log2(max(1, nbytes))))
        lst = self.free.setdefault(c, [])
        return lst.pop() if lst else self.torch.empty(c, dtype=self.torch.uint8).pin_memory()

    def put(self, t):
        self.free.setdefault(t.numel(), []).append(t)

    def reserve(self, sizes):
        """Allocates ahead (outside a timed region) what requests of these
        byte sizes would take at once."""
        need = {}
        for nbytes in sizes:
            c = 1 << max(12, math.ceil(math.log2(max(1, nbytes))))
            need[c] = need.get(c, 0) + 1
        for c, k in need.items():
            lst = self.free.setdefault(c, [])
            while len(lst) < k:
                lst.append(self.torch.empty(c, dtype=self.torch.uint8).pin_memory())


class RegroupService:
    """The continuous-batching servers of the three kernels (loom_b200.serving)."""

    def __init__(self, api, torch, stream, pool, inputs, profile=False):
        from loom_b200 import scenes as S
        from loom_b200 import serving

        self.api, self.pool, self.inputs = api, pool, inputs
        st = stream
        mk = dict(stream=st, profile=profile)
        self.p = serving.Pool(
            {
                "pt": api.Server(
                    "sphere_pt_f32", ring_threads=1 << 26, max_requests=512, slice_rounds=4,
                    forms=["instance", "local_iota"], header_words=S.HEADER_WORDS, reloc_word=4,
                    table_words=1 << 20, **regroup_opts("sphere_pt_f32", "batch"), **mk,
                ),
                "collatz": api.Server(
                    "collatz_u64", ring_threads=1 << 25, max_requests=512, slice_rounds=2,
                    **{**regroup_opts("collatz_u64"), "population": 1 << 22}, **mk,
                ),
                "fib": api.Server(
                    "fib_u64", ring_threads=1 << 23, max_requests=512, slice_rounds=2,
                    **{**regroup_opts("fib_u64"), "population": 1 << 21}, **mk,
                ),
            }
        )
        self.bufs = {}

    def device_bytes(self):
        return sum(s["device_bytes"] for s in self.p.stats().values())

    def submit(self, req):
        kind, n, a, _ = req
        info = self.p.servers[kind].info
        ob = [np.dtype(api_np(self.api, t)).itemsize for _, t in info.outputs]
        buf = self.pool.get(n * sum(ob))
        outs, off = [], buf.data_ptr()
        for b in ob:
            outs.append(off)
            off += n * b
        if kind == "pt":
            key = self.p.submit(kind, n, outputs=outs, **a)
        else:
            key = self.p.submit(kind, n, inputs=[self.inputs[kind][a : a + n]], outputs=outs)
        self.bufs[key] = buf
        return key

    def busy(self):
        return self.p.busy()

    def step(self):
        done = self.p.step()
        for key in done:
            self.p.result(*key)
            self.pool.put(self.bufs.pop(key))
        return done

    def lane_efficiency(self):
        ti = sum(s["thread_instr"] for s in self.p.stats().values())
        wi = sum(s["warp_instr"] for s in self.p.stats().values())
        return ti / (32.0 * wi) if wi else None

    def close(self):
        self.p.close()


def api_np(api, t):
    return api.NP_TYPE[t]


class PlainQueue:
    """The baseline: a FIFO queue per kernel; each step launches every
    waiting request of a kernel in one plain-engine launch (host columns in
    and out), and a request that arrives meanwhile waits for the next."""

    CAPACITY = {"pt": 1 << 27, "collatz": 1 << 25, "fib": 1 << 23}  # threads per launch

    def __init__(self, api, torch, stream, pool, inputs, profile=False):
        self.api, self.inputs = api, inputs
        self.pool = None
        self.f = {
            k: api.Function(v, self.CAPACITY[k], "plain", profile=profile) for k, v in SERVE_KERNELS.items()
        }
        self.wait = {k: [] for k in SERVE_KERNELS}
        self.t = 0

    def submit(self, req):
        self.t += 1
        self.wait[req[0]].append((self.t, req))
        return (req[0], self.t)

    def busy(self):
        return any(self.wait.values())

    def step(self):
        from loom_b200 import scenes as S

        api = self.api
        done = []
        for kind, lst in self.wait.items():
            if not lst:
                continue
            k, total = 0, 0
            while k < len(lst) and total + lst[k][1][1] <= self.CAPACITY[kind]:
                total += lst[k][1][1]
                k += 1
            batch, self.wait[kind] = lst[:k], lst[k:]
            if kind == "pt":
                table, starts = S.pack([r[3] for _, r in batch])
                n = int(starts[-1])
                self.f[kind].launch_host([api.Instance(), api.LocalIota()], n, instance_starts=starts, table=table)
            else:
                x = np.concatenate([self.inputs[kind][r[2] : r[2] + r[1]].numpy().view(np.uint64) for _, r in batch])
                self.f[kind](x)
            done += [(kind, t) for t, _ in batch]
        return done

    def device_bytes(self):
        return None

    def lane_efficiency(self):
        ti = wi = 0
        for f in self.f.values():
            s = f.stats()
            ti += s["thread_instr"]
            wi += s["warp_instr"]
        return ti / (32.0 * wi) if wi else None

    def close(self):
        for f in self.f.values():
            f.close()


OUT_BYTES = {"pt": 12, "collatz": 4, "fib": 8}


def run_requests(svc, reqs, arrivals):
    """Feeds `reqs` at `arrivals` (seconds from start) and steps `svc` until
    every request completed.  Returns (latencies, makespan, threads)."""
    if getattr(svc, "pool", None) is not None:
        svc.pool.reserve([r[1] * OUT_BYTES[r[0]] for r in reqs])
    t0 = time.perf_counter()
    i, lat, inflight = 0, [], {}
    last = 0.0
    while i < len(reqs) or inflight:
        now = time.perf_counter() - t0
        while i < len(reqs) and arrivals[i] <= now:
            inflight[svc.submit(reqs[i])] = arrivals[i]
            i += 1
        if inflight:
            for key in svc.step():
                last = time.perf_counter() - t0
                lat.append(last - inflight.pop(key))
        elif i < len(reqs):
            time.sleep(max(0.0, min(arrivals[i] - now, 0.002)))
    threads = sum(r[1] for r in reqs)
    return np.asarray(lat), last, threads


def serve_main(args, warmup, world, rank, local):
    import torch

    if world > 1:
        torch.cuda.set_device(local)
    from loom_b200 import api
    from loom_b200 import inputs as I

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    pool = PinnedPool(torch)
    inputs = {
        k: torch.from_numpy(I.uniform_int(20 + j, n, lo, hi).view(np.int64)).pin_memory()
        for j, (k, (n, lo, hi)) in enumerate(SERVE_POOL.items())
    }
    mix = ServeMix(seed=17 + rank)
    loads = (0.25, 0.5, 0.75, 1.0)
    out = {}
    with ClockSampler(local) as clk:
        for name, cls in (("regroup", RegroupService), ("plain", PlainQueue)):
            svc = cls(api, torch, stream, pool, inputs)
            # warm-up and capacity: a closed batch (every request at t = 0)
            run_requests(svc, mix.draw(24), np.zeros(24))
            cal = mix.draw(160)
            lat, span, threads = run_requests(svc, cal, np.zeros(len(cal)))
            cap = threads / span
            mean_threads = threads / len(cal)
            res = {"capacity_msamples_s": round(cap / 1e6, 3), "device_bytes": svc.device_bytes(), "loads": []}
            for L in loads:
                rate = L * cap / mean_threads  # requests per second
                count = max(8, int(rate * args.serve_seconds))
                reqs = mix.draw(count)
                arr = np.cumsum(mix.rng.exponential(1.0 / rate, size=count))
                lat, span, threads = run_requests(svc, reqs, arr)
                res["loads"].append(
                    {
                        "offered_load": L,
                        "requests": count,
                        "msamples_s": round(threads / span / 1e6, 3),
                        "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 2),
                        "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 2),
                        "mean_ms": round(float(lat.mean()) * 1e3, 2),
                    }
                )
            svc.close()
            # lane efficiency of the same mix in a counted (slower) run
            svc = cls(api, torch, stream, pool, inputs, profile=True)
            reqs = mix.draw(48)
            run_requests(svc, reqs, np.zeros(len(reqs)))
            le = svc.lane_efficiency()
            res["lane_efficiency"] = None if le is None else round(le, 4)
            svc.close()
            out[name] = res

    full = out["regroup"]["loads"][-1]
    line = base_line(
        args, warmup, world,
        "serving: Poisson arrivals at 25/50/75/100 % of measured capacity; mix 60 % render requests "
        "(batched-workload distribution), 20 % Collatz batches 2^16-2^22, 20 % Fibonacci batches 2^16-2^20",
        "sphere_pt_f32+collatz_u64+fib_u64", "mixed", "Msamples/s at 100 % offered load, p50/p99 latency",
        {"budget_bytes": SERVE_BUDGET, "seconds_per_load": args.serve_seconds},
    )
    line.update(
        {
            "value": full["msamples_s"],
            "p50_ms": full["p50_ms"],
            "p99_ms": full["p99_ms"],
            "fraction_of_capacity": round(full["msamples_s"] / out["regroup"]["capacity_msamples_s"], 4),
            "regroup": out["regroup"],
            "plain": out["plain"],
            "gpu_launches": None,
            "clocks": clk.summary(),
        }
    )
    if rank == 0:
        print(json.dumps(line))
        if args.csv:
            append_csv(args.csv, line)


def tune_main(args) -> None:
    """Coordinate search over the regrouping options (loom_b200.autotune) on
    this workload; writes the best point and the fastest points to a JSON
    file (merged into loom_b200/tuning.json by the maintainer)."""
    import torch

    from loom_b200 import api
    from loom_b200 import autotune as T

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    w = make_workload(args.workload)
    w.device_buffers(torch)
    f = api.Function(w.kernel, 0, "regroup")
    w.opts = regroup_opts(w.kernel, w.tune_key)
    space = dict(T.SPACE)
    if w.kernel == "sphere_pt_f32":  # 2 x 2832 queue bytes per thread in flight
        space["population"] = [p for p in space["population"] if p <= 1 << 22]

    def make_launch(opts):
        f.set_opts("regroup", **opts)
        return lambda: w.launch(f, api, stream)

    def validate():
        f.stats(raise_on_device_error=True)
        f.reset_stats()

    seed = [
        dict(T.DEFAULT, **regroup_opts(w.kernel, w.tune_key)),
        dict(T.DEFAULT, cost_model=True, utr_lanes=4, burst=32),
        dict(T.DEFAULT),
        # no parking: every live lane runs every burst (latency-bound runs
        # of few long threads)
        dict(T.DEFAULT, utr_lanes=1, spread_lanes=1, burst=64, period=1 << 20),
    ]
    res = T.tune(make_launch, w.n, seed=seed, space=space, budget_s=args.tune_budget,
                 log=lambda m: print(m, file=sys.stderr, flush=True), validate=validate)
    res["workload"] = args.workload
    res["kernel"] = w.kernel
    res["device"] = torch.cuda.get_device_name(0)
    pathlib.Path(args.tune).write_text(json.dumps(res, indent=1) + "\n")
    print(json.dumps({k: res[k] for k in ("kernel", "workload", "best", "ms", "msamples_s")}))
    f.close()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="pt", choices=["pt", "pt_small", "batch", "collatz", "fib", "loom_pt", "loom_pt2", "loom_pt_512", "loom_pt2_512", "loom_primary", "loom_primary_b20", "serve"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU leg (timing and parity)")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="serve: open-loop seconds per load")
    ap.add_argument("--tune", metavar="OUT", help="autotune the regrouping options of the workload, write JSON to OUT")
    ap.add_argument("--tune-budget", type=float, default=300.0, help="seconds of tuning")
    ap.add_argument("--csv", metavar="PATH", help="append a CSV row of the result to PATH")
    args = ap.parse_args()
    warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.workload == "serve":
        serve_main(args, warmup, world, rank, local)
        return
    if args.tune:
        tune_main(args)
        return

    w = make_workload(args.workload)
    w.opts = regroup_opts(w.kernel, w.tune_key)
    extra = {
        "threads_per_gpu": w.n,
        "l2": "outputs larger than L2 (no flush)",
        "regroup_options": w.opts,
        "regroup_options_from": "loom_b200/tuning.json (bench.py --tune, coordinate search)",
    }

    if args.impl == "reference":
        if rank != 0:
            return
        vals, info = [], None
        for i in range(warmup + args.steps):
            v, info, _ = cpu_reference(w, target_s=2.0)
            if i >= warmup:
                vals.append(v)
        value = statistics.median(vals)
        line = base_line(args, warmup, args.gpus, w.desc, w.kernel, w.dtype, METRIC, extra)
        line = {"impl": "reference", **line, "value": round(value, 3)}
        # the whole workload at the sampled rate
        line["ms_per_step"] = round(w.n / (value * 1e6) * 1e3, 4)
        line["cpu_baseline"] = dict(info, value=round(value, 3))
        line["e2e"] = {"value": round(value, 3), "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        print(json.dumps(line))
        if args.csv:
            append_csv(args.csv, line)
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
    tids = w.check_tids()

    res = {}
    for mode in ("plain", "regroup"):
        opts = dict(w.opts, graph=True) if mode == "regroup" else {}
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
        res[mode] = dict(ms=ms, stats=st, fn=f, out=w.outputs_at(tids))

    # the headline: the regrouping engine, clocks sampled during the timed region
    f = res["regroup"]["fn"]
    with ClockSampler(local) as clk:
        ms_r = time_steps(lambda: w.launch(f, api, stream), args.steps, warmup, torch, dist)
    st_r = f.stats(raise_on_device_error=True)
    kern_ms = st_r["ms"]
    out_r = w.outputs_at(tids)

    # the other tuned form of the same workload, when there is one: Loom's
    # majority rule with the cost model (the highest lane efficiency)
    alt = None
    from loom_b200 import autotune as T

    alt_opts = T.tuned(w.kernel, w.tune_key + "_majority") if w.tune_key != "default" else None
    if alt_opts:
        fa = api.Function(w.kernel, 0, "regroup", **dict(alt_opts, graph=True))
        ms_a = time_steps(lambda: w.launch(fa, api, stream), args.steps, warmup, torch, dist) / args.steps
        fa.set_opts("regroup", profile=True, **alt_opts)
        w.launch(fa, api, stream)
        torch.cuda.synchronize()
        sa = fa.stats(raise_on_device_error=True)
        alt = {
            "options": alt_opts,
            "value": round(world * w.n / (ms_a / 1e3) / 1e6, 3),
            "ms_per_step": round(ms_a, 4),
            "lane_efficiency": round(sa["lane_efficiency"], 4),
            "speedup_vs_plain": None,
            "same_outputs": bool(same_bits(w.outputs_at(tids), out_r)),
        }
        fa.close()

    e2e_s, e2e_ok, h2d, d2h = w.e2e(api, torch, args.steps, warmup, dist)
    e2e_s = max_over_ranks(e2e_s, dist)

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

    traffic, issue = ncu_rooflines(
        w, kern_ms, clk.summary().get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    )

    cpu, parity = None, {"sample_threads": int(len(tids)), "checked_against": None}
    plain_regroup_same = same_bits(res["plain"]["out"], out_r)
    parity["plain_equals_regroup"] = bool(plain_regroup_same)
    parity["e2e_equals_device"] = bool(e2e_ok)
    if not args.no_cpu:
        v, info, want = cpu_reference(w, check_tids=tids)
        cpu = dict(info, value=round(v, 3))
        parity["checked_against"] = info["kind"]
        parity["regroup_ok"] = bool(same_bits(out_r, want, w.kernel))
        parity["plain_ok"] = bool(same_bits(res["plain"]["out"], want, w.kernel))
        if w.kernel in ULP_TOLERANCE:
            parity["float_tolerance_ulp"] = ULP_TOLERANCE[w.kernel]

    line = base_line(args, warmup, world, w.desc, w.kernel, w.dtype, METRIC, extra)
    line.update(
        {
            "value": round(value, 3),
            "ms_per_step": round(ms_step, 4),
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
                "graph_launches": int(st_r.get("graph_launches", 0)),
            },
            "speedup_regroup_vs_plain": round(plain_ms / ms_step, 4),
            "regroup_majority_cost_model": (
                dict(alt, speedup_vs_plain=round(plain_ms / alt["ms_per_step"], 4)) if alt else None
            ),
            "lane_efficiency_note": "VM instructions executed / (32 x VM instructions issued per warp), in-kernel counters of a profiled launch",
            "parity": parity,
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
            "issue_roofline": issue,
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
    )
    print(json.dumps(line))
    if args.csv:
        append_csv(args.csv, line)
    for r in res.values():
        r["fn"].close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
