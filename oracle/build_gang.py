"""Recipe: the CPU gang port (Loom's compact and hybrid methods restated for
g++) into oracle/_lib/libloomgang.so.

BASELINE INFRASTRUCTURE ONLY.  Generates one C++ file per kernel of
loom_b200/ir/ (oracle/gang_emit.py) into oracle/_lib/gang/, compiles them
with oracle/gang_engine.hpp and links the library.  Needs only the committed
IR: no Loom headers.

Flags: the x86-64 level of the host CPUs (AVX-512), no FMA contraction
(every Loom instruction rounds on its own, as in bse), fused loom::fma as
bse's -mfma build has it, and -fno-math-errno so that square roots and
roundings vectorise (errno is not part of Loom's semantics; the values are
the IEEE ones either way, as clang's elementwise builtins in Loom's own SIMD
backend give them).
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = HERE / "_lib" / "libloomgang.so"
GEN = HERE / "_lib" / "gang"

FLAGS = [
    "-std=c++20",
    "-O3",
    "-march=x86-64-v4",
    "-mtune=native",
    "-mprefer-vector-width=512",
    "-fno-exceptions",
    "-ffp-contract=off",
    "-fno-fast-math",
    "-fno-math-errno",
    "-fno-trapping-math",
    "-mfma",
    "-fPIC",
    "-pthread",
    "-w",
]


def build(force: bool = False, jobs: int | None = None) -> pathlib.Path:
    import importlib.util

    sys.path.insert(0, str(ROOT))
    from loom_b200.codegen import ir

    # by path: run as a script, `oracle` on sys.path is oracle/oracle.py
    spec = importlib.util.spec_from_file_location("oracle_gang_emit", HERE / "gang_emit.py")
    gang_emit = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gang_emit)

    GEN.mkdir(parents=True, exist_ok=True)
    deps = [HERE / "gang_engine.hpp", HERE / "gang_emit.py", ROOT / "loom_b200" / "codegen" / "emit_cuda.py"]
    dep_mtime = max(d.stat().st_mtime for d in deps)
    stamp = GEN / "flags.txt"
    if not stamp.exists() or stamp.read_text() != " ".join(FLAGS):
        force = True
        stamp.write_text(" ".join(FLAGS))

    def one(name):
        src = GEN / f"{name}.cpp"
        text = gang_emit.generate(ir.load(name))
        if not src.exists() or src.read_text() != text:
            src.write_text(text)
        obj = GEN / f"{name}.o"
        if force or not obj.exists() or max(dep_mtime, src.stat().st_mtime) > obj.stat().st_mtime:
            _run(["g++", *FLAGS, f"-I{HERE}", "-c", str(src), "-o", str(obj)])
        return obj

    names = ir.available()
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(one, names))
    objs.append(_dispatcher(names, force))
    if force or not OUT.exists() or max(o.stat().st_mtime for o in objs) > OUT.stat().st_mtime:
        _run(["g++", "-shared", "-pthread", "-o", str(OUT), *map(str, objs)])
    return OUT


def _dispatcher(names, force: bool) -> pathlib.Path:
    """loom_gang_run(name, ...): the kernel's entry point by name."""
    lines = ["// Generated by oracle/build_gang.py: the gang port's entry by kernel name.", "#include <cstring>", ""]
    sig = ("const void* const* in, void* const* out, unsigned long long n, int threads, const unsigned* table, "
           "int method, unsigned stream, unsigned utr_den, unsigned long long* stats")
    for n in names:
        lines.append(f'extern "C" int loom_gang_run_{n}({sig});')
    lines += ["", f'extern "C" int loom_gang_run(const char* name, {sig})', "{"]
    for n in names:
        lines.append(f'    if(!std::strcmp(name, "{n}")) return loom_gang_run_{n}(in, out, n, threads, table, method, stream, utr_den, stats);')
    lines += ["    return -1;", "}", ""]
    src = GEN / "dispatch.cpp"
    text = "\n".join(lines)
    if not src.exists() or src.read_text() != text:
        src.write_text(text)
    obj = GEN / "dispatch.o"
    if force or not obj.exists() or src.stat().st_mtime > obj.stat().st_mtime:
        _run(["g++", *FLAGS, "-c", str(src), "-o", str(obj)])
    return obj


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"gang port build failed: {' '.join(cmd[-3:])}\n{r.stderr[-4000:]}")


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
