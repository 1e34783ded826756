"""Generates the golden fixtures tests/golden/<kernel>.npz.

Each fixture holds seeded input columns (tests/kernel_domains.py) and the
outputs of Loom's own scalar backend, vm::bse::function<K>, compiled from the
Loom headers into oracle/_ref/libloomref.so (oracle/build_ref.py).  Run it
where the Loom headers are available:

    python tests/golden/make_golden.py

The fixtures pin the C restatement (oracle/loom_interp.c) and the CUDA
engines on machines that have neither the Loom headers nor a compiler for
them.
"""

from __future__ import annotations

import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

from oracle import build_ref  # noqa: E402
from oracle import oracle as O  # noqa: E402
import kernel_domains as D  # noqa: E402

SEED = 20261203
SIZES = {"fib_u64": 4096, "collatz_u64": 4096}
DEFAULT_N = 1024


def _ir_io(name: str):
    ins, outs = [], []
    for ln in (O.IR_DIR / f"{name}.lir").read_text().splitlines():
        t = ln.split()
        if t and t[0] == "input":
            ins.append(t[2])
        elif t and t[0] == "output":
            outs.append(t[2])
    return ins, outs


def make_pt(name: str) -> pathlib.Path:
    """Path tracer fixtures: a small Cornell-box render and a batch of three
    random-scene requests in one launch, with their table and instance
    offsets."""
    import numpy as np

    from loom_b200 import scenes as S

    rng = np.random.default_rng(SEED)
    reqs = [S.cornell_request(32, 24, 4, seed=11)]
    for k in range(3):
        r = S.random_request(rng, seed=100 + k)
        r.width, r.height, r.spp = 16, 16, 4
        reqs.append(r)
    table, starts = S.pack(reqs)
    n = int(starts[-1])
    ins = O.expand_inputs(["instance", "local_iota"], n, starts, ["u32", "u32"])
    outs = O.ref_run(name, ins, n, threads=4, table=table)
    arrays = {f"in{i}": a for i, a in enumerate(ins)}
    arrays.update({f"out{j}": a for j, a in enumerate(outs)})
    arrays["table"] = table
    arrays["starts"] = starts
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    return path


def loom_pt_pixels(width: int = 40, height: int = 40):
    """Every pixel of a Loom path-tracer render, encoded as Loom's demo does
    (x << 16 | y, src/smallpt/vm/enc.hpp:30-34), in row order."""
    import numpy as np

    x, y = np.meshgrid(np.arange(width, dtype=np.uint32), np.arange(height, dtype=np.uint32))
    return ((x << 16) | y).reshape(-1)


def make(name: str) -> pathlib.Path:
    if name.startswith("sphere_pt"):
        return make_pt(name)
    if name.startswith(("pt_const", "pt2_const", "primary_const")):
        side = int(name.rsplit("_", 1)[1])
        ins = [loom_pt_pixels(side, side)]
        if len(ins[0]) > 4096:  # a seeded subset of the larger renders
            ins = D.inputs_for(name, 4096, SEED, ["u32"])
        outs = O.ref_run(name, ins, len(ins[0]), threads=8)
        arrays = {"in0": ins[0]}
        arrays.update({f"out{j}": a for j, a in enumerate(outs)})
        path = HERE / f"{name}.npz"
        np.savez_compressed(path, **arrays)
        return path
    ins_t, _ = _ir_io(name)
    n = SIZES.get(name, DEFAULT_N)
    ins = D.inputs_for(name, n, SEED, ins_t)
    if name == "fib_u64":
        # every n of the workload range appears at least once
        ins[0][:94] = np.arange(94, dtype=np.uint64)
    if name == "collatz_u64":
        ins[0][:8] = np.array([1, 2, 3, 6, 7, 27, 97, 837799], dtype=np.uint64)
    outs = O.ref_run(name, ins, n, threads=4)
    arrays = {f"in{i}": a for i, a in enumerate(ins)}
    arrays.update({f"out{j}": a for j, a in enumerate(outs)})
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    return path


def main() -> None:
    if build_ref.build() is None:
        raise SystemExit("Loom headers not found: set LOOM_REF_DIR")
    from loom_b200.codegen import ir

    wanted = sys.argv[1:]
    for name in ir.available():
        if not wanted or name in wanted:
            print(make(name))


if __name__ == "__main__":
    main()
