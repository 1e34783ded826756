"""Recipe: compile Loom's scalar backend (bse) into oracle/_ref/libloomref.so.

TEST AND BASELINE INFRASTRUCTURE ONLY.  Reads the Loom headers where they
lie (LOOM_REF_DIR, default ../reference beside this repository) and writes only into
oracle/_ref/ (per-kernel sources and objects in oracle/_ref/obj/).  g++ builds bse with -std=c++20 -fno-exceptions once Loom's
fast_float include is satisfied by a small forwarding shim
(loom_b200/frontend/shim); -ffp-contract=off keeps every Loom instruction a
separately rounded operation, as in Loom's own clang builds, where each
Compute is a statement of its own; -mfma makes loom::fma the fused
std::fma, as Loom's -march=native builds do on FMA hardware.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = HERE / "_ref" / "libloomref.so"


def ref_dir() -> pathlib.Path | None:
    env = os.environ.get("LOOM_REF_DIR")
    for c in ([pathlib.Path(env)] if env else []) + [ROOT.parent / "reference"]:
        if (c / "src" / "vm" / "bse.hpp").is_file():
            return c
    return None


FLAGS = [
    "-std=c++20",
    "-O3",
    # the x86-64 level of both host CPUs here (AVX-512 F/BW/CD/DQ/VL), tuned
    # for the build machine: the library is built once and runs on the GPU
    # machine's host too, so it must not use extensions only one of them has
    "-march=x86-64-v4",
    "-mtune=native",
    "-fno-exceptions",
    "-ffp-contract=off",
    "-fno-fast-math",
    # loom::fma is std::fma only when __FMA__ is defined (Loom
    # src/common/math.hpp:40-52); Loom's own builds use -march=native,
    # which defines it on every FMA-capable x86 (and the GPU uses fmaf).
    "-mfma",
    "-fPIC",
    "-pthread",
    "-w",
    # Loom's own path tracers nest type lists thousands deep
    "-ftemplate-depth=16384",
    "-fconstexpr-depth=16384",
    "-fconstexpr-ops-limit=4000000000",
]


def _registry():
    sys.path.insert(0, str(ROOT))
    from loom_b200.build import registry_kernels

    return registry_kernels()


def build(force: bool = False, jobs: int | None = None) -> pathlib.Path | None:
    """One object per registry kernel (its bse instantiation), compiled in
    parallel into oracle/_ref/obj/, plus the dispatcher; linked into
    oracle/_ref/libloomref.so."""
    ref = ref_dir()
    if ref is None:
        return OUT if OUT.exists() else None
    obj_dir = OUT.parent / "obj"
    obj_dir.mkdir(parents=True, exist_ok=True)
    deps = [HERE / "ref_kernel.hpp", *(ROOT / "loom_b200" / "kernels").glob("*.hpp")]
    dep_mtime = max(d.stat().st_mtime for d in deps)
    # a change of compiler flags rebuilds every object
    stamp = obj_dir / "flags.txt"
    if not stamp.exists() or stamp.read_text() != " ".join(FLAGS):
        force = True
        stamp.write_text(" ".join(FLAGS))
    inc = [
        f"-I{ref / 'src'}",
        f"-I{ref / 'ext' / 'include'}",
        f"-I{ROOT / 'loom_b200' / 'frontend' / 'shim'}",
        f"-I{HERE}",
    ]

    def compile_one(item):
        name, ty = item
        src = obj_dir / f"{name}.cpp"
        text = (
            "// bse runner of one registry kernel (generated by oracle/build_ref.py).\n"
            '#include "ref_kernel.hpp"\n'
            f'extern "C" int loom_ref_run_{name}(const void* const* in, void* const* out, '
            "std::uint64_t n, int threads, const std::uint32_t* table)\n{\n"
            f"    loom_ref::run_kernel<{ty}>(in, out, n, threads, table);\n"
            "    return 0;\n}\n"
        )
        if not src.exists() or src.read_text() != text:
            src.write_text(text)
        obj = obj_dir / f"{name}.o"
        if force or not obj.exists() or max(dep_mtime, src.stat().st_mtime) > obj.stat().st_mtime:
            _run(["g++", *FLAGS, *inc, "-c", str(src), "-o", str(obj)])
        return obj

    kernels = _registry()
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(compile_one, kernels))
    disp = obj_dir / "ref_runner.o"
    if force or not disp.exists() or max(dep_mtime, (HERE / "ref_runner.cpp").stat().st_mtime) > disp.stat().st_mtime:
        _run(["g++", *FLAGS, *inc, "-c", str(HERE / "ref_runner.cpp"), "-o", str(disp)])
    objs.append(disp)
    if force or not OUT.exists() or max(o.stat().st_mtime for o in objs) > OUT.stat().st_mtime:
        _run(["g++", "-shared", "-pthread", "-o", str(OUT), *map(str, objs)])
    return OUT


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference build failed: {' '.join(cmd[-3:])}\n{r.stderr[-4000:]}")


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
