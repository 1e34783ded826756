"""Host-side logic of bench.py, on CPU: the max-over-ranks reduction of the
multi-GPU run (two gloo ranks), the serving request mix and the option
lookup.  No GPU; the GPU arms are exercised on a B200."""

import os
import socket

import numpy as np
import pytest

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank's step time; every rank must see the slowest
        got = bench.max_over_ranks(10.0 + 3.5 * rank, dist, device="cpu")
        dist.barrier()
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=5) for _ in procs)
    assert res == {0: 13.5, 1: 13.5}


def test_max_over_ranks_single_process():
    assert bench.max_over_ranks(7.25) == 7.25


def test_serving_mix_is_seeded_and_follows_its_distribution():
    a = bench.ServeMix(17).draw(400)
    b = bench.ServeMix(17).draw(400)
    assert [(r[0], r[1]) for r in a] == [(r[0], r[1]) for r in b]
    kinds = [r[0] for r in a]
    assert 0.5 < kinds.count("pt") / len(kinds) < 0.7
    for kind, n, extra, _ in a:
        if kind == "collatz":
            assert 1 << 16 <= n <= 1 << 22 and n & (n - 1) == 0
            assert 0 <= extra <= bench.SERVE_POOL["collatz"][0] - n
        elif kind == "fib":
            assert 1 << 16 <= n <= 1 << 20
        else:
            assert n == extra["header"][0] * extra["header"][1] * (1 << extra["header"][2])


def test_regroup_options_come_from_the_tuning_file():
    from loom_b200 import autotune as T

    for kernel in bench.FALLBACK:
        o = bench.regroup_opts(kernel)
        assert o, kernel
        t = T.tuned(kernel)
        if t is not None:
            assert o == t


def test_reference_runner_without_gpu():
    """The CPU leg runs and checks on any machine: reference outputs of a
    few Collatz threads equal the known stopping times."""
    run, kind, cores = bench._reference_runner()
    x = np.array([1, 2, 3, 6, 7, 27], dtype=np.uint64)
    (steps,) = run("collatz_u64", [x], None)
    assert list(steps) == [0, 1, 7, 8, 16, 111]
    assert kind in ("reference", "port") and cores >= 1


def test_issue_roofline_of_the_committed_capture():
    """The headline bench line's issue roofline: the committed capture's
    SASS warp instructions per path, scaled to the full launch, over the
    kernel time, against 148 SMs x 4 schedulers at the sampled clock; only
    for the options the capture was taken with."""
    import json

    w = bench.make_workload("pt")
    cap = json.loads((bench.ROOT / "profiles" / "roofline_traffic.json").read_text())["pt"]
    w.opts = dict(cap["sass_options"])
    traffic, issue = bench.ncu_rooflines(w, 41.47, 1965.0)
    assert issue is not None
    per = issue["sass_warp_inst_per_thread"]
    want = per * w.n / 41.47e-3 / 1e9
    assert issue["achieved"] == pytest.approx(want, rel=1e-3)
    assert issue["peak"] == pytest.approx(148 * 4 * 1.965, abs=0.05)
    assert 0 < issue["frac"] < 1
    # another option set: no issue figure from a capture of different code
    w.opts = dict(w.opts, schedule=0)
    assert bench.ncu_rooflines(w, 41.47, 1965.0)[1] is None


def test_vm_issue_roofline():
    """The headline roofline: VM instructions executed (summed over Loom
    threads) per second against 32 lanes x 148 SMs x 4 schedulers x one
    warp instruction per cycle at the sampled clock."""
    r = bench.issue_roofline(6382 * 50331648, 41.44, 1965.0)
    assert r["peak"] == pytest.approx(32 * 148 * 4 * 1.965, rel=1e-4)
    assert r["achieved"] == pytest.approx(6382 * 50331648 / 41.44e-3 / 1e9, rel=1e-4)
    assert r["frac"] == pytest.approx(0.208, abs=0.002)


def test_rooflines_without_a_capture(tmp_path):
    w = bench.make_workload("collatz")
    w.opts = bench.regroup_opts(w.kernel, w.tune_key)
    assert bench.ncu_rooflines(w, 3.6, 1965.0) == (None, None)
    assert bench.ncu_rooflines(w, 3.6, 1965.0, path=tmp_path / "none.json") == (None, None)
    f = tmp_path / "t.json"
    f.write_text('{"default": {"kernel": "collatz_u64", "dram_bytes_per_thread": 12.5}}')
    traffic, issue = bench.ncu_rooflines(w, 3.6, 1965.0, path=f)
    assert traffic == int(12.5 * w.n) and issue is None


def test_csv_rows_of_bench_lines(tmp_path):
    """`--csv` appends one row per run, as Loom's benchmarks do
    (src/benchmarks/bm.hpp:103-139), with the GPU figures of the line."""
    import csv

    line = {
        "value": 1213.0, "ms_per_step": 41.49, "n_gpus": 1,
        "plain": {"value": 346.9}, "regroup": {"lane_efficiency": 0.4156},
        "roofline": {"achieved": 14.6}, "issue_roofline": {"frac": 0.7356},
        "config": {"workload": "sphere path tracer", "kernel": "sphere_pt_f32"},
    }
    serve = {"value": 1406.2, "p50_ms": 27.4, "p99_ms": 104.2, "n_gpus": 1, "regroup": {"lane_efficiency": 0.85},
             "config": {"workload": "serving", "kernel": "sphere_pt_f32+collatz_u64+fib_u64"}}
    ref = {"impl": "reference", "value": 9.0, "ms_per_step": 5580.0, "n_gpus": 1, "config": {"workload": "w", "kernel": "k"}}
    f = tmp_path / "runs.csv"
    for ln in (line, serve, ref):
        bench.append_csv(str(f), ln)
    rows = list(csv.DictReader(open(f)))
    assert [r["impl"] for r in rows] == ["b200", "b200", "reference"]
    assert list(rows[0]) == bench.CSV_FIELDS
    assert float(rows[0]["msamples_s"]) == 1213.0 and float(rows[0]["issue_frac"]) == 0.7356
    assert float(rows[0]["plain_msamples_s"]) == 346.9 and float(rows[0]["state_gbs"]) == 14.6
    assert float(rows[1]["p99_ms"]) == 104.2 and rows[1]["issue_frac"] == ""
    assert rows[2]["lane_efficiency"] == "" and rows[0]["date"].endswith("Z")


def test_reference_arm_under_torchrun_prints_one_line():
    """The reference arm launched as the multi-GPU bench is launched (two
    ranks under torch.distributed.run): rank 0 times Loom's CPU backend and
    prints the only line; the other rank exits 0 without work."""
    import json
    import subprocess
    import sys

    root = bench.ROOT
    cmd = [
        sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
        "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
        str(root / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3",
        "--workload", "collatz",
    ]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")


class _FibFull:
    """A workload stand-in for full_parity: 3000 Fibonacci threads."""

    kernel = "fib_u64"

    def __init__(self):
        from oracle import oracle as O

        self.n = 3000
        self.x = O.uniform_int(9, self.n, 0, 93).astype(np.uint64)

    def ref_inputs(self, tids):
        return [self.x[np.asarray(tids, dtype=np.int64)]], None


def test_full_parity_checks_every_thread():
    """full_parity runs bse on every thread and compares each kept engine's
    outputs bit for bit; one wrong output anywhere fails that engine."""
    from oracle import oracle as O

    if not O.ref_available():
        pytest.skip("Loom's bse not built here")
    w = _FibFull()
    good = O.val_fib(w.x)
    bad = good.copy()
    bad[2999] ^= np.uint64(1)
    res = {"regroup": {"full": [good]}, "plain": {"full": [bad]}}
    d = bench.full_parity(w, res)
    assert d["threads"] == 3000 and d["regroup_ok"] is True and d["plain_ok"] is False
    assert "full" not in res["regroup"]  # the host copies are released
