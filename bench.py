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
        self.spp = spp
        self.pixels = width * height
        self.table, self.starts = S.pack([self.req])
        self.n = self.req.threads
        self.desc = (
            f"sphere path tracer, Cornell box of 9 spheres (walls r=1e5, mirror, glass IOR 1.5, light), "
            f"{width}x{height} x {spp} spp = {self.n} threads, FP32, RR from depth 5, max depth 16; "
            f"output: the {width}x{height} RGB f32 image (per-pixel mean of its {spp} samples in sample order)"
        )
        self.in_bytes = 0
        self.out_bytes = 12

    def inputs(self, api):
        return [api.Broadcast(0, "u32"), api.Iota()]

    def device_buffers(self, torch):
        self.d_table = torch.from_numpy(self.table.view(np.int32)).cuda()
        self.d_out = [torch.empty(self.n, dtype=torch.float32, device="cuda") for _ in range(3)]
        self.d_img = [torch.empty(self.pixels, dtype=torch.float32, device="cuda") for _ in range(3)]

    def launch(self, f, api, stream):
        """One step: the render (one thread per pixel-sample), then the image
        (per-pixel means, loom_b200_group_mean)."""
        f.launch_device(self.inputs(api), self.d_out, self.n, table=self.d_table, stream=stream)
        for o, img in zip(self.d_out, self.d_img):
            api.group_mean(o, img, self.pixels, self.spp, stream=stream)

    launches_per_step = 5  # queue reset + megakernel (or the plain kernel) + 3 group means

    def check_tids(self):
        """Every sample of 256 random pixels (16,384 threads)."""
        rng = np.random.default_rng(5)
        px = np.sort(rng.choice(self.pixels, size=256, replace=False))
        return (px[:, None] * self.spp + np.arange(self.spp)[None, :]).reshape(-1)

    def image_rows_ok(self, want_samples, tids):
        """The device image at the checked pixels against the per-pixel mean
        (in sample order) of the reference's per-sample outputs."""
        import torch

        from loom_b200 import scenes as S

        px = np.asarray(tids, dtype=np.int64).reshape(-1, self.spp)[:, 0] // self.spp
        want = S.pixel_average(want_samples, self.spp)
        ix = torch.from_numpy(px).cuda()
        got = np.stack([img[ix].cpu().numpy() for img in self.d_img], axis=1)
        return bool(np.array_equal(got.view(np.uint32), want.view(np.uint32)))

    def ref_inputs(self, tids):
        tids = np.asarray(tids, dtype=np.uint64)
        return [np.zeros(len(tids), dtype=np.uint32), tids.astype(np.uint32)], self.table

    def e2e(self, api, torch, steps, warmup, dist):
        """The image through loom_b200_launch_host_mean: scene table in,
        render, per-pixel means, image rows back to pinned host memory."""
        h_img = [torch.empty(self.pixels, dtype=torch.float32).pin_memory() for _ in range(3)]
        fe = api.Function(self.kernel, self.n, "regroup", **self.opts)

        def step():
            fe.launch_host_mean(self.inputs(api), self.n, group=self.spp, table=self.table, outputs=h_img)

        for _ in range(warmup):
            step()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        dt = time.perf_counter() - t0
        ok = all(torch.equal(h, d.cpu()) for h, d in zip(h_img, self.d_img))
        fe.close()
        return dt, ok, self.table.nbytes, 3 * 4 * self.pixels


class BatchedPathTracing(PathTracing):
    """Many render requests of uneven size in one launch: each request has
    its own resolution, sample count and random scene (loom_b200.scenes
    .random_request); threads of all requests share the megakernel and are
    mapped to (request, sample) on the device from the instance offsets."""

    tune_key = "batch"
    launches_per_step = 2

    def __init__(self, count=256, seed=3):
        from loom_b200 import scenes as S

        rng = np.random.default_rng(seed)
        self.reqs = [S.random_request(rng, seed=i + 1) for i in range(count)]
        self.table, self.starts = S.pack(self.reqs)
        self.n = int(self.starts[-1])
        self.spp_of = np.array([r.spp for r in self.reqs], dtype=np.uint32)
        self.pixels = int(sum(r.width * r.height for r in self.reqs))
        self.desc = (
            f"{count} batched render requests (seed {seed}): resolution from {{64,128,256,512}}^2, spp from "
            f"{{1,4,16,64}}, 8-64 random spheres each (60/20/20 diffuse/mirror/glass, 1-4 emitters), "
            f"{self.n} threads in one launch, FP32; end to end: each request's image (per-pixel means)"
        )
        self.in_bytes = 0
        self.out_bytes = 12

    def inputs(self, api):
        return [api.Instance(), api.LocalIota()]

    def device_buffers(self, torch):
        self.d_table = torch.from_numpy(self.table.view(np.int32)).cuda()
        self.d_out = [torch.empty(self.n, dtype=torch.float32, device="cuda") for _ in range(3)]
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

    def request_of(self, tids):
        return np.searchsorted(self.starts, np.asarray(tids, dtype=np.uint64), side="right") - 1

    def image_rows_ok(self, want_samples, tids):
        return None

    def ref_inputs(self, tids):
        tids = np.asarray(tids, dtype=np.uint64)
        inst = (np.searchsorted(self.starts, tids, side="right") - 1).astype(np.int64)
        return [inst.astype(np.uint32), (tids - self.starts[inst]).astype(np.uint32)], self.table

    def e2e(self, api, torch, steps, warmup, dist):
        """Every request's image through loom_b200_launch_host_mean (per
        request: its samples per pixel), compared with the per-pixel means
        of the device's per-sample outputs."""
        h_img = [torch.empty(self.pixels, dtype=torch.float32).pin_memory() for _ in range(3)]
        fe = api.Function(self.kernel, self.n, "regroup", **self.opts)

        def step():
            fe.launch_host_mean(self.inputs(api), self.n, instance_group=self.spp_of, instance_starts=self.starts,
                                table=self.table, outputs=h_img)

        for _ in range(warmup):
            step()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        dt = time.perf_counter() - t0
        # check: the images of 8 requests against the means of the device outputs
        from loom_b200 import scenes as S

        ok, row = True, 0
        for i, r in enumerate(self.reqs):
            rows = r.width * r.height
            if i % 32 == 0:
                a, b = int(self.starts[i]), int(self.starts[i + 1])
                want = S.pixel_average([o[a:b].cpu().numpy() for o in self.d_out], r.spp)
                got = np.stack([h[row : row + rows].numpy() for h in h_img], axis=1)
                ok &= bool(np.array_equal(got.view(np.uint32), want.view(np.uint32)))
            row += rows
        fe.close()
        return dt, ok, self.table.nbytes + self.starts.nbytes, 3 * 4 * self.pixels


class IntegerLoop(Workload):
    launches_per_step = 2

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
    launches_per_step = 2

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
        "Loom bse (vm::bse::function), g++ -O3 -march=x86-64-v4 -mfma -ffp-contract=off, one std::thread per core"
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


def cpu_hybrid_port(w, target_s: float = 2.0, stream: int = 288, utr_den: int = 16):
    """Loom's hybrid method on all host cores, as the gang port restates it
    (oracle/gang_engine.hpp: N-lane gangs, threaded dispatch, counting sort
    by PC, one stream of `stream` threads per worker in the manner of
    mp::Shop; Loom's best published path-tracer configuration is a stream of
    288 and a 1/16 threshold, site-docs/bm-results.md:40).  Timed like
    cpu_reference on a bounded random sample (seed 7); checked bit for bit
    against bse on the first 1024 of those threads.  None when the port is
    not built."""
    from oracle import oracle as O

    if not O.gang_available():
        return None
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(7)
    pool = rng.integers(0, w.n, size=min(w.n, 1 << 26))
    m = 1 << 12
    while True:
        ins, table = w.ref_inputs(pool[:m])
        t0 = time.perf_counter()
        O.gang_run(w.kernel, ins, len(ins[0]), threads=cores, table=table, stream=stream, utr_den=utr_den)
        dt = time.perf_counter() - t0
        if dt > target_s / 8 or m >= len(pool):
            break
        m = min(len(pool), m * 4)
    m = min(len(pool), max(m, int(m * target_s / max(dt, 1e-9))))
    ins, table = w.ref_inputs(pool[:m])
    st = {}
    t0 = time.perf_counter()
    got = O.gang_run(w.kernel, ins, len(ins[0]), threads=cores, table=table, stream=stream, utr_den=utr_den,
                     stats=st)
    dt = time.perf_counter() - t0
    k = min(1024, len(ins[0]))
    ok = None
    if O.ref_available():
        want = O.ref_run(w.kernel, [a[:k] for a in ins], k, threads=cores, table=table)
        ok = bool(same_bits([g[:k] for g in got], want, w.kernel))
    from loom_b200.codegen import ir as _ir
    from oracle import gang_emit

    lanes = gang_emit.lanes_of(_ir.load(w.kernel))
    return {
        "value": round(m / dt / 1e6, 3),
        "unit": "Msamples/s",
        "cores": cores,
        "kind": "port",
        "method": f"hybrid stream, {stream} threads per worker, threshold 1/{utr_den}, {lanes}-lane gangs",
        "lane_efficiency": round(st["lanes"] / max(1, st["blocks"] * lanes), 4),
        "sample": f"{m} threads drawn at random (seed 7) from the workload's {w.n}, on {_cpu_model()}; Loom's "
                  "hybrid method restated for g++ (oracle/gang_engine.hpp), one worker per core",
        "seconds": round(dt, 3),
        "equals_bse_on_first_1024": ok,
    }


# Float outputs that pass through the host libm's sinf/cosf (Loom's
# pt2_const) are held within this many ulp of the reference; everything else
# is compared bit for bit.
# A libm value one ulp apart is carried through the rest of the path's
# arithmetic: at 512x512 about 0.4 % of pixels differ, by at most 14 ulp.
ULP_TOLERANCE = {"pt2_const_40": 16, "pt2_const_512": 16}
IMAGE_RMSE_TOLERANCE = 1e-6  # relative RMSE of each float output (radiance channel) as an image


def same_bits(got, want, kernel: str = "") -> bool:
    for g, w in zip(got, want):
        g, w = np.ascontiguousarray(g), np.ascontiguousarray(w)
        if kernel in ULP_TOLERANCE and w.dtype.kind == "f":
            ulps = np.abs(g.astype(np.float64) - w.astype(np.float64)) / np.spacing(np.abs(w)).astype(np.float64)
            if len(w) and float(ulps.max()) > ULP_TOLERANCE[kernel]:
                return False
            w64 = w.astype(np.float64)
            ref = float(np.sqrt(np.mean(w64 * w64))) if len(w) else 0.0
            if ref > 0 and float(np.sqrt(np.mean((g.astype(np.float64) - w64) ** 2))) / ref > IMAGE_RMSE_TOLERANCE:
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

    overlap = True  # start the busy servers' slices together (one round each)

    def __init__(self, api, torch, stream, pool, inputs, profile=False):
        from loom_b200 import scenes as S
        from loom_b200 import serving

        self.api, self.pool, self.inputs = api, pool, inputs
        # one stream per server, one device-memory budget for all
        self.streams = {k: torch.cuda.Stream() for k in SERVE_KERNELS}
        self.budget = api.Budget(SERVE_BUDGET)
        mk = dict(profile=profile, budget=self.budget)
        # the servers' own tuned options ("serve": the options of short
        # slices, which are not those of one long launch); collatz and fib
        # servers run 256-thread CTAs, so that one CTA of each fits on an SM
        # beside one 512-thread CTA of the path tracer (512 x 64 + 256 x 40 +
        # 256 x 48 registers: 54 K of the SM's 64 K)
        self.p = serving.Pool(
            {
                "pt": api.Server(
                    "sphere_pt_f32", ring_threads=1 << 26, max_requests=512, slice_rounds=4,
                    forms=["instance", "local_iota"], header_words=S.HEADER_WORDS, reloc_word=4,
                    table_words=1 << 20, **regroup_opts("sphere_pt_f32", "serve"), stream=self.streams["pt"], **mk,
                ),
                "collatz": api.Server(
                    "collatz_u64", ring_threads=1 << 25, max_requests=512, slice_rounds=2,
                    **{**regroup_opts("collatz_u64", "serve"), "population": 1 << 22, "block_size": 256, "ctas_per_sm": 0},
                    stream=self.streams["collatz"], **mk,
                ),
                "fib": api.Server(
                    "fib_u64", ring_threads=1 << 23, max_requests=512, slice_rounds=2,
                    **{**regroup_opts("fib_u64"), "population": 1 << 21, "block_size": 256, "ctas_per_sm": 0},
                    stream=self.streams["fib"], **mk,
                ),
            },
            shared_ctas={"pt": 1, "collatz": 1, "fib": 1} if self.overlap else None,
        )
        self.bufs = {}
        self.reqs = {}
        self.keep_samples = False
        self.samples = []  # (kind, reference inputs, table, outputs) of sampled threads

    def device_bytes(self):
        return sum(s["device_bytes"] for s in self.p.stats().values())

    def _sample(self, key, req, buf):
        """Keeps 4 threads of a completed request (their reference inputs and
        the served outputs) for the parity check."""
        from loom_b200 import scenes as S

        kind, n, a, r = req
        rng = np.random.default_rng(len(self.samples))
        j = np.unique(rng.integers(0, n, size=4))
        info = self.p.servers[kind].info
        dts = [np.dtype(api_np(self.api, t)) for _, t in info.outputs]
        host = buf.numpy()
        got, off = [], 0
        for dt in dts:
            col = host[off : off + n * dt.itemsize].view(dt)
            got.append(col[j].copy())
            off += n * dt.itemsize
        if kind == "pt":
            table, _ = S.pack([r])
            ins = [np.zeros(len(j), dtype=np.uint32), j.astype(np.uint32)]
        else:
            table = None
            ins = [self.inputs[kind][a : a + n].numpy().view(np.uint64)[j]]
        self.samples.append((kind, ins, table, got))

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
        self.reqs[key] = req
        return key

    def busy(self):
        return self.p.busy()

    def step(self):
        done = self.p.step()
        for key in done:
            self.p.result(*key)
            req = self.reqs.pop(key)
            buf = self.bufs.pop(key)
            if self.keep_samples and key[1] % 4 == 0:
                self._sample(key, req, buf)
            self.pool.put(buf)
        return done

    def lane_efficiency(self):
        ti = sum(s["thread_instr"] for s in self.p.stats().values())
        wi = sum(s["warp_instr"] for s in self.p.stats().values())
        return ti / (32.0 * wi) if wi else None

    def slice_times(self):
        """(summed slice time, time any slice ran) so far, in ms, from the
        slices' global-timer intervals."""
        return self.p.slice_ns / 1e6, self.p.union_ns / 1e6

    def budget_waits(self):
        return sum(s["budget_waits"] for s in self.p.stats().values())

    def close(self):
        self.p.close()


class RegroupServiceSerial(RegroupService):
    """The same servers stepped one after the other (each slice with the
    whole GPU and its own slice length)."""

    overlap = False


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


def serve_measure(seconds: float, rank: int = 0, local: int = 0, parity: bool = False):
    """The serving loop of both services (continuous-batching regroup
    servers, plain FIFO queue) under Poisson arrivals at 25/50/75/100 % of
    each one's measured capacity, `seconds` of arrivals per load.  With
    `parity`, sampled threads of some completed requests of the regroup
    servers are kept for a check against the reference.  Returns (results
    per service, clock summary)."""
    import torch

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
        for name, cls in (("regroup", RegroupService), ("regroup_serial", RegroupServiceSerial), ("plain", PlainQueue)):
            svc = cls(api, torch, stream, pool, inputs)
            # warm-up and capacity: a closed batch (every request at t = 0)
            run_requests(svc, mix.draw(24), np.zeros(24))
            cal = mix.draw(160)
            lat, span, threads = run_requests(svc, cal, np.zeros(len(cal)))
            cap = threads / span
            mean_threads = threads / len(cal)
            res = {"capacity_msamples_s": round(cap / 1e6, 3), "device_bytes": svc.device_bytes(), "loads": []}
            if parity and name == "regroup":
                svc.keep_samples = True
            for L in loads:
                rate = L * cap / mean_threads  # requests per second
                count = max(8, int(rate * seconds))
                reqs = mix.draw(count)
                arr = np.cumsum(mix.rng.exponential(1.0 / rate, size=count))
                t_0 = svc.slice_times() if hasattr(svc, "slice_times") else None
                lat, span, threads = run_requests(svc, reqs, arr)
                row = {
                    "offered_load": L,
                    "requests": count,
                    "msamples_s": round(threads / span / 1e6, 3),
                    "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 2),
                    "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 2),
                    "mean_ms": round(float(lat.mean()) * 1e3, 2),
                }
                if t_0 is not None:
                    # the slices' device time summed over servers, against the
                    # time during which any slice ran: above 1 when slices of
                    # different kernels ran on the GPU together
                    t_1 = svc.slice_times()
                    row["slices_ms"] = round(t_1[0] - t_0[0], 1)
                    row["any_slice_ms"] = round(t_1[1] - t_0[1], 1)
                    row["wall_ms"] = round(span * 1e3, 1)
                    row["overlap"] = round((t_1[0] - t_0[0]) / max(1e-9, t_1[1] - t_0[1]), 3)
                res["loads"].append(row)
            if parity and name == "regroup":
                res["parity"] = serve_parity(svc, inputs)
            if hasattr(svc, "budget_waits"):
                res["budget"] = {"limit_bytes": svc.budget.limit, "requests_that_waited": svc.budget_waits(),
                                 "admission": "n x (state_size + column bytes per thread) + table bytes, "
                                              "shared by the three servers, arrival order"}
            svc.close()
            # lane efficiency of the same mix in a counted (slower) run
            svc = cls(api, torch, stream, pool, inputs, profile=True)
            reqs = mix.draw(48)
            run_requests(svc, reqs, np.zeros(len(reqs)))
            le = svc.lane_efficiency()
            res["lane_efficiency"] = None if le is None else round(le, 4)
            svc.close()
            out[name] = res
    return out, clk.summary()


def serve_parity(svc, inputs):
    """Sampled threads of completed requests (every request whose ticket is
    a multiple of 4, 4 threads each) against the reference."""
    run, kind, _ = _reference_runner()
    ok, checked, reqs = True, 0, set()
    for kind_, want_ins, table, got in svc.samples:
        want = run(SERVE_KERNELS[kind_], want_ins, table)
        ok &= same_bits(got, want, SERVE_KERNELS[kind_])
        checked += len(got[0])
    return {"checked_against": kind, "requests_checked": len(svc.samples), "threads_checked": checked,
            "ok": bool(ok)}


def serve_main(args, warmup, world, rank, local):
    import torch

    if world > 1:
        torch.cuda.set_device(local)
    out, clocks = serve_measure(args.serve_seconds, rank, local)
    full = out["regroup_serial"]["loads"][-1]
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
            "fraction_of_capacity": round(full["msamples_s"] / out["regroup_serial"]["capacity_msamples_s"], 4),
            "regroup_serial": out["regroup_serial"],
            "regroup_overlapping": out["regroup"],
            "plain": out["plain"],
            "gpu_launches": None,
            "clocks": clocks,
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
    space["max_regs"] = api.reg_caps(w.kernel)  # the caps compiled for this kernel

    def make_launch(opts):
        f.set_opts("regroup", **opts)
        return lambda: w.launch(f, api, stream)

    def validate():
        f.stats(raise_on_device_error=True)
        f.reset_stats()

    constraint = None
    if args.tune_min_lane_eff:
        def constraint(opts):
            """One counted launch: VM-level lane efficiency of the point."""
            f.set_opts("regroup", profile=True, **opts)
            w.launch(f, api, stream)
            le = f.stats(raise_on_device_error=True)["lane_efficiency"]
            f.reset_stats()
            return le >= args.tune_min_lane_eff

    seed = [
        dict(T.DEFAULT, **regroup_opts(w.kernel, w.tune_key)),
        dict(T.DEFAULT, cost_model=True, utr_lanes=4, burst=32),
        dict(T.DEFAULT),
        # no parking: every live lane runs every burst (latency-bound runs
        # of few long threads)
        dict(T.DEFAULT, utr_lanes=1, spread_lanes=1, burst=64, period=1 << 20),
    ]
    if args.tune_seed:
        seed.insert(0, dict(T.DEFAULT, **json.loads(args.tune_seed)))
    res = T.tune(make_launch, w.n, seed=seed, space=space, budget_s=args.tune_budget,
                 log=lambda m: print(m, file=sys.stderr, flush=True), validate=validate,
                 constraint=constraint)
    res["constraint"] = {"min_lane_efficiency": args.tune_min_lane_eff} if constraint else None
    res["workload"] = args.workload
    res["kernel"] = w.kernel
    res["device"] = torch.cuda.get_device_name(0)
    pathlib.Path(args.tune).write_text(json.dumps(res, indent=1) + "\n")
    print(json.dumps({k: res[k] for k in ("kernel", "workload", "best", "ms", "msamples_s")}))
    f.close()


def measure(w, api, torch, stream, steps, warmup, dist, tids, forms, clocks_for=None, full_for=()):
    """The plain engine and each regrouping form of workload `w`: CUDA-event
    time of `steps` steps after `warmup`, one counted launch (VM-instruction
    counters, lane efficiency) and the outputs at `tids`.  `forms` maps a
    name to regrouping options; the form named `clocks_for` is timed again
    with the clocks sampled; the engines and forms named in `full_for` keep
    every output of their last timed step (host arrays, "full").  Returns a
    dict per engine and form."""
    res = {}
    for name, mode, opts in [("plain", "plain", {})] + [(k, "regroup", o) for k, o in forms.items()]:
        run_opts = dict(opts, graph=True) if mode == "regroup" else {}
        f = api.Function(w.kernel, 0, mode, **run_opts)
        clk = None
        if name == clocks_for:
            with ClockSampler(torch.cuda.current_device()) as c:
                ms = time_steps(lambda: w.launch(f, api, stream), steps, warmup, torch, dist)
            clk = c.summary()
        else:
            ms = time_steps(lambda: w.launch(f, api, stream), steps, warmup, torch, dist)
        st_t = f.stats(raise_on_device_error=True)
        out = w.outputs_at(tids)
        extra = {}
        if name in full_for:
            extra["full"] = [o.cpu().numpy() for o in w.d_out]
        if hasattr(w, "image_rows_ok"):
            extra["image"] = [img[:].clone() for img in getattr(w, "d_img", [])]
        dev_bytes = f.device_bytes()
        f.reset_stats()
        f.set_opts(mode, profile=True, **run_opts)  # one counted launch
        w.launch(f, api, stream)
        torch.cuda.synchronize()
        st = f.stats(raise_on_device_error=True)
        f.close()
        res[name] = dict(ms=ms / steps, kernel_ms=st_t["ms"], stats=st, out=out, opts=opts, clocks=clk,
                         device_bytes=dev_bytes, rounds=st_t["rounds"] / max(1, st_t["launches"]),
                         parks=st_t["parks"] / max(1, st_t["launches"]),
                         state_bytes=st_t["state_bytes"] / max(1, st_t["launches"]), **extra)
    return res


def regroup_forms(w):
    """The tuned regrouping forms of a workload: the fastest (the headline
    form) and, where tuned, Loom's majority rule with the cost model and the
    lane-efficiency form (the fastest one measured at >= 70 % SASS lane
    efficiency)."""
    from loom_b200 import autotune as T

    forms = {"regroup": w.opts}
    if w.tune_key != "default":
        for key, name in (("_majority", "majority_cost_model"), ("_lane", "lane_efficiency_form")):
            o = T.tuned(w.kernel, w.tune_key + key)
            if o:
                forms[name] = o
    return forms


def issue_roofline(vm_instr: float, kern_ms: float, sm_mhz: float) -> dict:
    """The SIMT issue roofline of a launch: VM instructions executed (summed
    over Loom threads) per second against 32 lanes x 148 SMs x 4 schedulers
    x one warp instruction per cycle at the sampled SM clock."""
    got = vm_instr / (kern_ms / 1e3) / 1e9
    top = 32 * 148 * 4 * sm_mhz / 1e3
    return {"achieved": round(got, 1), "peak": round(top, 1), "unit": "G VM thread-instructions/s",
            "frac": round(got / top, 4)}


def workload_summary(w, res, world, cpu=None, want=None, e2e=None, tids=None, full=None):
    """The figures of one workload: value and ms per step of the tuned
    regrouping form, the plain engine and the other forms beside it, lane
    efficiencies, parity against the reference on the sampled threads."""
    rg, pl = res["regroup"], res["plain"]
    d = {
        "workload": w.desc,
        "kernel": w.kernel,
        "threads": w.n,
        "value": round(world * w.n / (rg["ms"] / 1e3) / 1e6, 3),
        "unit": "Msamples/s",
        "ms_per_step": round(rg["ms"], 4),
        "lane_efficiency": round(rg["stats"]["lane_efficiency"], 4),
        "regroup_options": rg["opts"],
        "device_bytes": rg["device_bytes"],
        "plain": {
            "value": round(world * w.n / (pl["ms"] / 1e3) / 1e6, 3),
            "ms_per_step": round(pl["ms"], 4),
            "lane_efficiency": round(pl["stats"]["lane_efficiency"], 4),
        },
        "speedup_vs_plain": round(pl["ms"] / rg["ms"], 4),
    }
    if rg["opts"].get("plain_below", 0) > w.n:
        # the tuner measured that the persistent megakernel does not pay for
        # this workload: the regrouping handle runs it on the plain engine
        d["engine_used"] = "plain (regrouping handle's plain_below rule, set by the tuner)"
    for name, r in res.items():
        if name in ("plain", "regroup"):
            continue
        d[name] = {
            "options": r["opts"],
            "value": round(world * w.n / (r["ms"] / 1e3) / 1e6, 3),
            "ms_per_step": round(r["ms"], 4),
            "lane_efficiency": round(r["stats"]["lane_efficiency"], 4),
            "speedup_vs_plain": round(pl["ms"] / r["ms"], 4),
            "same_outputs": bool(same_bits(r["out"], rg["out"])),
            "device_bytes": r["device_bytes"],
        }
    par = {"sample_threads": int(len(tids)), "plain_equals_regroup": bool(same_bits(pl["out"], rg["out"]))}
    if want is not None:
        par["checked_against"] = cpu["kind"]
        par["regroup_ok"] = bool(same_bits(rg["out"], want, w.kernel))
        par["plain_ok"] = bool(same_bits(pl["out"], want, w.kernel))
        for name, r in res.items():
            if name not in ("plain", "regroup"):
                par[f"{name}_ok"] = bool(same_bits(r["out"], want, w.kernel))
        if w.kernel in ULP_TOLERANCE:
            par["float_tolerance_ulp"] = ULP_TOLERANCE[w.kernel]
            par["image_relative_rmse_tolerance"] = IMAGE_RMSE_TOLERANCE
        if hasattr(w, "request_of"):
            req = w.request_of(tids)
            bad = set()
            for g, x in zip(rg["out"], want):
                diff = np.ascontiguousarray(g).view(np.uint8).reshape(len(tids), -1) != np.ascontiguousarray(
                    x).view(np.uint8).reshape(len(tids), -1)
                bad |= set(int(r) for r in req[diff.any(axis=1)])
            par["requests_checked"] = int(len(np.unique(req)))
            par["threads_per_request"] = 4
            par["requests_failed"] = sorted(bad)
        if rg.get("image") and hasattr(w, "image_rows_ok"):
            w.d_img = rg["image"]
            par["image_ok"] = w.image_rows_ok(want, tids)
            par["image_pixels_checked"] = int(len(tids) // getattr(w, "spp", 1))
    if full is not None:
        par["full_size"] = full
    full_ok = all(v for k, v in (full or {}).items() if k.endswith("_ok"))
    par["parity"] = bool(par.get("regroup_ok", par["plain_equals_regroup"]) and par["plain_equals_regroup"]
                         and par.get("image_ok", True) is not False and not par.get("requests_failed")
                         and full_ok)
    d["parity"] = par
    if cpu is not None:
        d["cpu_baseline"] = cpu
    if e2e is not None:
        d["e2e"] = e2e
    return d


def run_e2e(w, api, torch, steps, warmup, dist, world):
    e2e_s, ok, h2d, d2h = w.e2e(api, torch, steps, warmup, dist)
    e2e_s = max_over_ranks(e2e_s, dist)
    return {
        "value": round(world * w.n * steps / e2e_s / 1e6, 3),
        "unit": "Msamples/s",
        "h2d_bytes_per_step": int(h2d),
        "d2h_bytes_per_step": int(d2h),
        "equals_device": bool(ok),
    }


def sub_config(name, api, torch, stream, steps, warmup, dist, world, no_cpu, extra_check=None, full_check=False):
    """One more configuration of the default run, measured like the
    headline with its own (smaller) step count; with `full_check`, every
    output is checked against bse (full_parity)."""
    w = make_workload(name)
    w.opts = regroup_opts(w.kernel, w.tune_key)
    w.device_buffers(torch)
    tids = w.check_tids()
    full_for = ("regroup", "plain") if full_check and not no_cpu else ()
    res = measure(w, api, torch, stream, steps, warmup, dist, tids, regroup_forms(w), full_for=full_for)
    e2e = run_e2e(w, api, torch, steps, warmup, dist, world)
    cpu = want = full = None
    if not no_cpu:
        v, info, want = cpu_reference(w, check_tids=tids, target_s=1.0)
        cpu = dict(info, value=round(v, 3))
        if full_for:
            full = full_parity(w, res)
    d = workload_summary(w, res, world, cpu, want, e2e, tids, full)
    if not no_cpu:
        d["cpu_hybrid_port"] = cpu_hybrid_port(w, target_s=1.0)
    d["steps"], d["warmup"] = steps, warmup
    if extra_check:
        d["parity"].update(extra_check(w))
        d["parity"]["parity"] = bool(d["parity"]["parity"] and all(
            v for k, v in d["parity"].items() if k.endswith("_ok") and isinstance(v, bool)))
    for attr in ("d_out", "d_in", "d_table", "d_starts", "d_img"):
        if hasattr(w, attr):
            delattr(w, attr)
    torch.cuda.empty_cache()
    return d


def full_parity(w, res, names=("regroup", "plain")):
    """Every output of the full workload against Loom's bse, run on all host
    cores over every thread: the last timed step's outputs of the engines
    and forms in `names` (kept by measure(full_for=...)), bit for bit (float
    outputs through libm sin/cos within the stated ulp and image bounds),
    and, for the path tracer, every pixel of the device image against the
    per-pixel means of bse's samples in sample order."""
    from oracle import oracle as O

    if not O.ref_available():
        return None
    cores = os.cpu_count() or 1
    ins, table = w.ref_inputs(np.arange(w.n, dtype=np.int64))
    t0 = time.perf_counter()
    want = O.ref_run(w.kernel, ins, w.n, threads=cores, table=table)
    dt = time.perf_counter() - t0
    d = {"threads": int(w.n), "reference": "Loom bse on every thread", "reference_seconds": round(dt, 3),
         "cores": cores}
    for name in names:
        if res.get(name, {}).get("full") is not None:
            d[f"{name}_ok"] = bool(same_bits(res[name]["full"], want, w.kernel))
    if res["regroup"].get("image") and hasattr(w, "spp"):
        from loom_b200 import scenes as S

        img = np.stack([c.cpu().numpy() for c in res["regroup"]["image"]], axis=1)
        d["image_ok"] = bool(np.array_equal(img.view(np.uint32), S.pixel_average(want, w.spp).view(np.uint32)))
        d["image_pixels"] = int(img.shape[0])
    for name in names:
        res.get(name, {}).pop("full", None)
    return d


def fib_full_check(w):
    """Every one of the 2^20 Fibonacci outputs against Loom's validator
    (val_fib, src/tests/programs.hpp:353-368)."""
    from oracle import oracle as O

    got = w.d_out[0].cpu().numpy().view(np.uint64)
    return {"all_threads_vs_val_fib_ok": bool(np.array_equal(got, O.val_fib(w.x))), "all_threads": int(w.n)}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="pt", choices=["pt", "pt_small", "batch", "collatz", "fib", "loom_pt", "loom_pt2", "loom_pt_512", "loom_pt2_512", "loom_primary", "loom_primary_b20", "serve"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU leg (timing and parity)")
    ap.add_argument("--only", metavar="FORM", default="",
                    help="time one engine or form alone (plain, regroup, majority_cost_model, "
                         "lane_efficiency_form): no counted launch, no end-to-end leg, no CPU leg (for profilers)")
    ap.add_argument("--form-opts", default="", metavar="JSON",
                    help="with --only: options merged into the form's tuned ones")
    ap.add_argument("--no-configs", action="store_true",
                    help="pt: skip the other configurations (fib, collatz, batch, serve) of the default run")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="serve: open-loop seconds per load")
    ap.add_argument("--tune", metavar="OUT", help="autotune the regrouping options of the workload, write JSON to OUT")
    ap.add_argument("--tune-budget", type=float, default=300.0, help="seconds of tuning")
    ap.add_argument("--tune-min-lane-eff", type=float, default=0.0,
                    help="tune: only points whose counted VM lane efficiency reaches this are eligible")
    ap.add_argument("--tune-seed", default="", help="tune: JSON options of an extra seed point")
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
        vals, secs, info = [], [], None
        for i in range(warmup + args.steps):
            v, info, _ = cpu_reference(w, target_s=2.0)
            if i >= warmup:
                vals.append(v)
                secs.append(info["seconds"])
        value = statistics.median(vals)
        line = base_line(args, warmup, args.gpus, w.desc, w.kernel, w.dtype, METRIC, extra)
        line = {"impl": "reference", **line, "value": round(value, 3)}
        # each step times a bounded random sample of the workload; ms_per_step
        # is the sampled step's own time, the whole workload's projection beside it
        line["ms_per_step"] = round(1e3 * statistics.median(secs), 4)
        line["ms_per_step_note"] = (
            "wall time of one step, which runs a random sample of the workload's threads (cpu_baseline.sample); "
            "projected_ms_full_workload is the whole workload at the sampled rate"
        )
        line["projected_ms_full_workload"] = round(w.n / (value * 1e6) * 1e3, 4)
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

    forms = regroup_forms(w)
    if args.only:
        # one engine or form, W + K launches and nothing else: the launch
        # sequence a profiler's -s/-c counts refer to
        opts = {} if args.only == "plain" else dict(forms[args.only], **json.loads(args.form_opts or "{}"))
        f = api.Function(w.kernel, 0, "plain" if args.only == "plain" else "regroup", **opts)
        ms = time_steps(lambda: w.launch(f, api, stream), args.steps, warmup, torch, dist)
        st = f.stats(raise_on_device_error=True)
        f.close()
        if rank == 0:
            print(json.dumps({"workload": w.desc, "form": args.only, "options": opts,
                              "ms_per_step": round(ms / args.steps, 4), "kernel_ms": round(st["ms"], 4),
                              "value": round(world * w.n / (ms / args.steps / 1e3) / 1e6, 3)}))
        return
    full_for = ("regroup", "plain") if rank == 0 and not args.no_cpu and args.workload == "pt" else ()
    res = measure(w, api, torch, stream, args.steps, warmup, dist, tids, forms, clocks_for="regroup",
                  full_for=full_for)
    rg = res["regroup"]
    clocks = rg["clocks"]
    e2e = run_e2e(w, api, torch, args.steps, warmup, dist, world)

    cpu = want = hyb = full = None
    if rank == 0 and not args.no_cpu:
        v, info, want = cpu_reference(w, check_tids=tids)
        cpu = dict(info, value=round(v, 3))
        hyb = cpu_hybrid_port(w)
        if full_for:
            full = full_parity(w, res)
    summary = workload_summary(w, res, world, cpu, want, e2e, tids, full)

    # the other configurations of the default run, each with its parity check
    configs = {}
    if args.workload == "pt" and not args.no_configs:
        for attr in ("d_out", "d_img", "d_table"):
            if hasattr(w, attr):
                delattr(w, attr)
        torch.cuda.empty_cache()
        configs["fib"] = sub_config("fib", api, torch, stream, args.steps, warmup, dist, world, args.no_cpu,
                                    fib_full_check)
        configs["collatz"] = sub_config("collatz", api, torch, stream, args.steps, warmup, dist, world,
                                        args.no_cpu, full_check=True)
        configs["batch"] = sub_config("batch", api, torch, stream, max(2, args.steps // 4), 3, dist, world,
                                      args.no_cpu)
        # Loom's own path tracers at 512x512 (where the tuner found that the
        # megakernel does not pay and set the regrouping handle's plain rule)
        for name in ("loom_pt_512", "loom_pt2_512"):
            configs[name] = sub_config(name, api, torch, stream, 3, 3, dist, world, args.no_cpu, full_check=True)
        sv, sv_clk = serve_measure(1.0, rank, local, parity=not args.no_cpu)
        full = sv["regroup_serial"]["loads"][-1]
        configs["serve"] = {
            "workload": "serving: Poisson arrivals at 25/50/75/100 % of measured capacity (1 s per load); mix "
                        "60 % render requests (batched-workload distribution), 20 % Collatz batches 2^16-2^22, "
                        "20 % Fibonacci batches 2^16-2^20; 100 GB thread-state budget shared by the servers",
            "value": full["msamples_s"],
            "unit": "Msamples/s at 100 % offered load (regrouping servers stepped one after the other)",
            "p50_ms": full["p50_ms"],
            "p99_ms": full["p99_ms"],
            "fraction_of_capacity": round(full["msamples_s"] / sv["regroup_serial"]["capacity_msamples_s"], 4),
            "regroup_serial": sv["regroup_serial"],
            "regroup_overlapping": sv["regroup"],
            "plain": sv["plain"],
            "parity": sv["regroup"].pop("parity", None),
            "clocks": sv_clk,
        }
        torch.cuda.set_stream(stream)

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
    sm_mhz = (clocks or {}).get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)

    kern_ms = rg["kernel_ms"]
    vm_instr = rg["stats"]["thread_instr"]  # one counted launch: VM instructions summed over threads
    roof = issue_roofline(vm_instr, kern_ms, sm_mhz)
    traffic, sass = ncu_rooflines(w, kern_ms, sm_mhz)
    # algorithmic bytes of one megakernel launch: inputs, outputs, table and
    # the queue state the engine moved (saves + restores, counted in-kernel)
    algo_bytes = w.n * (w.in_bytes + w.out_bytes) + rg["state_bytes"]
    hbm = algo_bytes / (kern_ms / 1e3) / 1e9
    roof.update(
        {
            "bound": "simt_issue",
            "vm_instructions_per_launch": int(vm_instr),
            "vm_instructions_per_thread": round(vm_instr / w.n, 1),
            "kernel_ms": round(kern_ms, 4),
            "sm_mhz": sm_mhz,
            "peak_source": "32 lanes x 148 SMs x 4 schedulers x 1 warp instruction per cycle at the sampled SM clock",
            "traffic": traffic,
            "hbm": {
                "achieved": round(hbm, 2),
                "peak": hbm_peak,
                "unit": "GB/s",
                "frac": round(hbm / hbm_peak, 5),
                "algorithmic_bytes": int(algo_bytes),
                "traffic": traffic,
                "peak_source": peak_src,
            },
            "note": "VM instructions = Loom Compute/Jump/ParmJump executed, summed over Loom threads, counted "
                    "in-kernel; the issue roofline in SASS warp instructions and the DRAM traffic come from the "
                    "ncu capture named in profiles/roofline_traffic.json",
        }
    )
    roof = {"bound": roof.pop("bound"), **roof}

    line = base_line(args, warmup, world, w.desc, w.kernel, w.dtype, METRIC, extra)
    line.update(
        {
            "value": summary["value"],
            "ms_per_step": summary["ms_per_step"],
            "plain": summary["plain"],
            "regroup": {
                "kernel_ms": round(kern_ms, 4),
                "lane_efficiency": summary["lane_efficiency"],
                "rounds": int(rg["rounds"]),
                "parks_per_thread": round(rg["parks"] / w.n, 4),
                "state_bytes_per_launch": int(rg["state_bytes"]),
                "device_bytes": int(rg["device_bytes"]),
            },
            "speedup_regroup_vs_plain": summary["speedup_vs_plain"],
            "lane_efficiency_note": "VM instructions executed / (32 x VM instructions issued per warp), in-kernel "
                                    "counters of a profiled launch; the SASS-level figure (ncu) in sass_issue",
            "parity": summary["parity"],
            "roofline": roof,
            "sass_issue": sass,
            "cpu_baseline": cpu,
            "cpu_hybrid_port": hyb,
            "e2e": {k: v for k, v in e2e.items() if k != "equals_device"},
            "gpu_launches": w.launches_per_step * args.steps,
            "clocks": clocks,
        }
    )
    for k in ("majority_cost_model", "lane_efficiency_form"):
        if k in summary:
            line[k] = summary[k]
    line["parity"]["e2e_equals_device"] = e2e["equals_device"]
    if configs:
        line["configs"] = configs
    print(json.dumps(line))
    if args.csv:
        append_csv(args.csv, line)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
