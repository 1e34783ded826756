"""Recipe: compile Loom's scalar backend (bse) into oracle/_ref/libloomref.so.

TEST AND BASELINE INFRASTRUCTURE ONLY.  Reads the Loom headers where they
lie (LOOM_REF_DIR, default /root/reference) and writes only into
oracle/_ref/.  g++ builds bse with -std=c++20 -fno-exceptions once Loom's
fast_float include is satisfied by a small forwarding shim
(loom_b200/frontend/shim); -ffp-contract=off keeps every Loom instruction a
separately rounded operation, as in Loom's own clang builds, where each
Compute is a statement of its own; -mfma makes loom::fma the fused
std::fma, as Loom's -march=native builds do on FMA hardware.
"""

from __future__ import annotations

import os
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = HERE / "_ref" / "libloomref.so"


def ref_dir() -> pathlib.Path | None:
    env = os.environ.get("LOOM_REF_DIR")
    for c in ([pathlib.Path(env)] if env else []) + [pathlib.Path("/root/reference")]:
        if (c / "src" / "vm" / "bse.hpp").is_file():
            return c
    return None


def build(force: bool = False) -> pathlib.Path | None:
    ref = ref_dir()
    if ref is None:
        return OUT if OUT.exists() else None
    srcs = [HERE / "ref_runner.cpp", *(ROOT / "loom_b200" / "kernels").glob("*.hpp")]
    if OUT.exists() and not force:
        if OUT.stat().st_mtime > max(s.stat().st_mtime for s in srcs):
            return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    cmd = [
        "g++",
        "-std=c++20",
        "-O2",
        "-fno-exceptions",
        "-ffp-contract=off",
        "-fno-fast-math",
        # loom::fma is std::fma only when __FMA__ is defined (Loom
        # src/common/math.hpp:40-52); Loom's own builds use -march=native,
        # which defines it on every FMA-capable x86 (and the GPU uses fmaf).
        "-mfma",
        "-fPIC",
        "-shared",
        "-pthread",
        "-w",
        "-ftemplate-depth=4096",
        "-fconstexpr-depth=4096",
        "-fconstexpr-ops-limit=1000000000",
        f"-I{ref / 'src'}",
        f"-I{ref / 'ext' / 'include'}",
        f"-I{ROOT / 'loom_b200' / 'frontend' / 'shim'}",
        str(HERE / "ref_runner.cpp"),
        "-o",
        str(OUT),
    ]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference build failed:\n{r.stderr[-4000:]}")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
