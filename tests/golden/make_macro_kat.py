"""Known answers for the macro kernels: Loom's plain C++ functions run on
the inputs of each kernel's golden fixture, written to
tests/golden/macro_kat.npz (32-bit words; float outputs as their bits).

  rotl32_u32, threefry_u32, canonical_f32, bump_u32   src/common/random.hpp
  cross_f32, norm_f32                                 src/common/linal.hpp

The golden outputs themselves come from Loom's scalar backend running the
VM macros (make_golden.py); tests/test_oracle.py checks them against these
answers as Loom's own tests do (src/tests/vm_smallpt.cpp:349-378: exact;
src/tests/vm_linal.cpp:82-156: within 30 ulp for 99 % of the inputs).
Compiled like the scalar backend's runner (-ffp-contract=off -mfma).

    python tests/golden/make_macro_kat.py     # needs the Loom headers and g++
"""

from __future__ import annotations

import os
import pathlib
import subprocess
import sys
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]

# kernel -> (function of macro_kat.cpp, output columns)
KERNELS = {
    "rotl32_u32": ("rotl32", 1),
    "threefry_u32": ("threefry", 2),
    "canonical_f32": ("canonical", 1),
    "bump_u32": ("bump", 2),
    "cross_f32": ("cross", 3),
    "norm_f32": ("norm", 3),
}


def ref_dir() -> pathlib.Path:
    for c in (os.environ.get("LOOM_REF_DIR"), str(pathlib.Path(__file__).resolve().parents[3] / "reference")):
        if c and (pathlib.Path(c) / "src" / "common" / "random.hpp").is_file():
            return pathlib.Path(c)
    raise SystemExit("Loom headers not found: set LOOM_REF_DIR")


def main() -> None:
    ref = ref_dir()
    with tempfile.TemporaryDirectory() as tmp:
        exe = pathlib.Path(tmp) / "macro_kat"
        subprocess.run(
            ["g++", "-std=c++20", "-O1", "-ffp-contract=off", "-mfma", f"-I{ref / 'src'}",
             f"-I{ref / 'ext' / 'include'}", f"-I{ROOT / 'loom_b200' / 'frontend' / 'shim'}",
             str(HERE / "macro_kat.cpp"), "-o", str(exe)],
            check=True,
        )
        arrays = {}
        for kernel, (fn, nout) in KERNELS.items():
            g = np.load(HERE / f"{kernel}.npz")
            ins = [g[k] for k in sorted(k for k in g.files if k.startswith("in"))]
            n = len(ins[0])
            stdin = b"".join(np.ascontiguousarray(a).view(np.uint32).tobytes() for a in ins)
            r = subprocess.run([str(exe), fn, str(n)], input=stdin, capture_output=True, check=True)
            outs = np.frombuffer(r.stdout, dtype=np.uint32).reshape(nout, n)
            for j in range(nout):
                arrays[f"{kernel}_out{j}"] = outs[j].copy()
        path = HERE / "macro_kat.npz"
        np.savez_compressed(path, **arrays)
        print(path)


if __name__ == "__main__":
    sys.exit(main())
