"""Build libloom_b200.so: IR extraction (optional), CUDA code generation and
nvcc compilation for sm_100a.

Steps
  1. extract  (only where the Loom headers are available, LOOM_REF_DIR or
              ../reference beside this repository): one small g++ program per registry kernel
              prints its IR; loom_b200/ir/*.lir are written for kernels that
              have none, for all with --reextract (after a kernel changed);
  2. generate loom_b200/csrc/gen/<kernel>.cu for every .lir file;
  3. compile  every .cu with nvcc -gencode arch=compute_100a,code=sm_100a and
              link loom_b200/libloom_b200.so.
Steps 2-3 need only this repository, so a machine without the Loom headers
rebuilds from the committed IR.  Compilation is incremental (mtime based).
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import re
import shutil
import subprocess
import sys
from typing import List, Optional

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
GEN = CSRC / "gen"
IR_DIR = PKG / "ir"
OBJ = ROOT / "_build" / "obj"
LIB = PKG / "libloom_b200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Float rounding must match Loom's scalar backend: no FMA contraction, IEEE
# division and square root, denormals kept.
FP_FLAGS = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "--expt-relaxed-constexpr",
    *ARCH,
    *FP_FLAGS,
    f"-I{INCLUDE}",
    f"-I{CSRC}",
]


def default_ref_dir() -> Optional[pathlib.Path]:
    env = os.environ.get("LOOM_REF_DIR")
    cands = [pathlib.Path(env)] if env else []
    cands.append(ROOT.parent / "reference")
    for c in cands:
        if (c / "src" / "vm" / "core.hpp").is_file():
            return c
    return None


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and pathlib.Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def run(cmd: List[str], **kw) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


# ---------------------------------------------------------------- 1. extract
# Deep template limits: Loom's larger kernels (its own path tracers) nest
# type lists thousands deep.
TEMPLATE_FLAGS = [
    "-ftemplate-depth=16384",
    "-fconstexpr-depth=16384",
    "-fconstexpr-ops-limit=4000000000",
]


def registry_kernels() -> List[tuple]:
    """(name, C++ type) of every X(name, type) line of the registry."""
    out = []
    for ln in (PKG / "kernels" / "registry.hpp").read_text().splitlines():
        m = re.match(r"\s*X\((\w+),\s*(.*?)\)\s*\\?\s*$", ln)
        if m:
            out.append((m.group(1), m.group(2).strip()))
    return out


def _write_if_changed(p: pathlib.Path, text: str) -> None:
    if not p.exists() or p.read_text() != text:
        p.write_text(text)


def extract(ref: pathlib.Path, names: Optional[List[str]] = None, jobs: Optional[int] = None) -> None:
    """Rebuild the text IR of the registry kernels from their Loom types: one
    small program per kernel (compiled in parallel, without optimisation, as
    it runs once) prints the kernel's IR."""
    work = ROOT / "_build" / "extract"
    work.mkdir(parents=True, exist_ok=True)
    deps = [PKG / "frontend" / "ir_emit.hpp", PKG / "frontend" / "b200_ops.hpp"]
    deps += list((PKG / "kernels").glob("*.hpp"))
    dep_mtime = max(d.stat().st_mtime for d in deps)
    IR_DIR.mkdir(exist_ok=True)
    todo = [(n, t) for n, t in registry_kernels() if not names or n in names]

    def one(item) -> None:
        name, ty = item
        src = work / f"{name}.cpp"
        exe = work / name
        _write_if_changed(
            src,
            "// IR extractor of one registry kernel (generated by loom_b200/build.py).\n"
            '#include "ir_emit.hpp"\n'
            '#include "registry.hpp"\n'
            "#include <fstream>\n"
            "int main(int argc, char* argv[])\n{\n"
            "    if(argc < 2) return 2;\n"
            "    std::ofstream f(argv[1]);\n"
            f'    f << loom::vm::b200::ir::emit<{ty}>("{name}");\n'
            "    return f ? 0 : 1;\n}\n",
        )
        if not exe.exists() or max(dep_mtime, src.stat().st_mtime) > exe.stat().st_mtime:
            run(
                [
                    "g++",
                    "-std=c++20",
                    "-O0",
                    "-fno-exceptions",
                    "-w",
                    *TEMPLATE_FLAGS,
                    f"-I{PKG / 'frontend'}",
                    f"-I{PKG / 'kernels'}",
                    f"-I{ref / 'src'}",
                    f"-I{ref / 'ext' / 'include'}",
                    f"-I{PKG / 'frontend' / 'shim'}",
                    str(src),
                    "-o",
                    str(exe),
                ]
            )
        tmp = work / f"{name}.lir"
        run([str(exe), str(tmp)])
        dst = IR_DIR / f"{name}.lir"
        if not dst.exists() or dst.read_text() != tmp.read_text():
            shutil.copyfile(tmp, dst)

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        list(ex.map(one, todo))


# ---------------------------------------------------------------- 2. generate
def generate() -> List[str]:
    sys.path.insert(0, str(ROOT))
    from loom_b200.codegen import emit_cuda, ir

    GEN.mkdir(parents=True, exist_ok=True)
    names = ir.available(IR_DIR)
    for n in names:
        k = ir.load(n, IR_DIR)
        _write_if_changed(GEN / f"{n}.cu", emit_cuda.generate(k))
    _write_if_changed(GEN / "registry.cu", emit_cuda.generate_registry(names))
    for stale in GEN.glob("*.cu"):
        if stale.stem not in names and stale.stem != "registry":
            stale.unlink()
    return names


# ---------------------------------------------------------------- 3. compile
def _headers() -> List[pathlib.Path]:
    return list((CSRC / "engine").glob("*.cuh")) + [
        CSRC / "runtime_iface.h",
        CSRC / "request_book.hpp",
        INCLUDE / "loom_b200.h",
    ]


def compile_all(jobs: Optional[int] = None, verbose: bool = False) -> pathlib.Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    srcs = [CSRC / "runtime.cu", CSRC / "server.cu", CSRC / "static_scratch.cu", *sorted(GEN.glob("*.cu"))]
    hdr_mtime = max(h.stat().st_mtime for h in _headers())
    cc = nvcc()

    def one(src: pathlib.Path) -> pathlib.Path:
        obj = OBJ / (src.stem + ".o")
        if obj.exists() and obj.stat().st_mtime > max(src.stat().st_mtime, hdr_mtime):
            return obj
        run([cc, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])
        if verbose:
            print(f"  nvcc {src.name}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(one, srcs))
    if not LIB.exists() or max(o.stat().st_mtime for o in objs) > LIB.stat().st_mtime:
        run([cc, "-shared", *ARCH, "-o", str(LIB), *map(str, objs), "-lcudart"])
    return LIB


def build(extract_ir: bool = True, verbose: bool = False, reextract: bool = False) -> pathlib.Path:
    """Extract the IR of registry kernels that have none yet (all of them
    with `reextract`, after a kernel's source changed), generate, compile."""
    ref = default_ref_dir() if extract_ir else None
    if ref is not None:
        names = None if reextract else [n for n, _ in registry_kernels() if not (IR_DIR / f"{n}.lir").exists()]
        if names is None or names:
            extract(ref, names)
    generate()
    return compile_all(verbose=verbose)


if __name__ == "__main__":
    print(build(verbose=True, reextract="--reextract" in sys.argv))
