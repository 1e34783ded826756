"""Recipe: build tests/cpp/_bin/vm_b200, the C++ front-end test.

TEST INFRASTRUCTURE ONLY.  The program includes Loom's own test headers and
kernel types, so it builds only where the Loom sources are (LOOM_REF_DIR, or
the default location probed by loom_b200.build); the binary links
loom_b200/libloom_b200.so through an $ORIGIN rpath and so runs wherever the
repository's built files are copied.
"""

from __future__ import annotations

import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / "_bin" / "vm_b200"


def build(force: bool = False) -> pathlib.Path | None:
    sys.path.insert(0, str(ROOT))
    from loom_b200.build import LIB, default_ref_dir

    ref = default_ref_dir()
    if ref is None:
        return OUT if OUT.exists() else None
    srcs = [
        HERE / "vm_b200.cpp",
        ROOT / "include" / "loom_b200.hpp",
        ROOT / "include" / "loom_b200.h",
        ROOT / "loom_b200" / "frontend" / "ir_emit.hpp",
        ROOT / "loom_b200" / "frontend" / "b200_ops.hpp",
    ]
    if OUT.exists() and not force and OUT.stat().st_mtime > max(s.stat().st_mtime for s in srcs):
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    cmd = [
        "g++",
        "-std=c++20",
        "-O1",
        "-fno-exceptions",
        "-w",
        "-ftemplate-depth=4096",
        "-fconstexpr-depth=4096",
        "-fconstexpr-ops-limit=1000000000",
        f"-I{ROOT / 'include'}",
        f"-I{ROOT / 'loom_b200' / 'frontend'}",
        f"-I{ref / 'src'}",
        f"-I{ref / 'ext' / 'include'}",
        f"-I{ROOT / 'loom_b200' / 'frontend' / 'shim'}",
        str(HERE / "vm_b200.cpp"),
        "-o",
        str(OUT),
        f"-L{LIB.parent}",
        "-lloom_b200",
        "-Wl,-rpath,$ORIGIN/../../../loom_b200",
    ]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"C++ front-end test build failed:\n{r.stderr[-6000:]}")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
