"""Oracle: CPU restatements of Loom's scalar semantics.

TEST AND BASELINE INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg use this module to check results against; the
product (loom_b200) never imports it.

Three layers, each pinned against the next:
  * ``Interp``  — oracle/loom_interp.c, a plain-C restatement of vm::bse
    (Loom src/vm/bse.hpp:400-649 and core.hpp:736-802) that runs the text IR;
  * ``ref_run`` — Loom's own bse compiled from its headers into
    oracle/_ref/libloomref.so (oracle/build_ref.py), available where it was
    built;
  * numpy reference functions restating Loom's test validators
    (src/tests/programs.hpp:290-389) and the workload definitions.
The golden fixtures under tests/golden/ were produced by ``ref_run`` and are
what the C restatement is checked against on machines without the Loom
headers.
"""

from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
INTERP_SRC = HERE / "loom_interp.c"
INTERP_SO = HERE / "_lib" / "libloominterp.so"
REF_SO = HERE / "_ref" / "libloomref.so"
IR_DIR = ROOT / "loom_b200" / "ir"

NP_TYPE = {
    "b8": np.uint8,
    "i8": np.int8,
    "u8": np.uint8,
    "i16": np.int16,
    "u16": np.uint16,
    "i32": np.int32,
    "u32": np.uint32,
    "i64": np.int64,
    "u64": np.uint64,
    "f32": np.float32,
    "f64": np.float64,
}


# ---------------------------------------------------------------- C port
def build_interp(force: bool = False) -> pathlib.Path:
    """Compile the C restatement (gcc, no FMA contraction)."""
    if INTERP_SO.exists() and not force:
        if INTERP_SO.stat().st_mtime > INTERP_SRC.stat().st_mtime:
            return INTERP_SO
    INTERP_SO.parent.mkdir(parents=True, exist_ok=True)
    cmd = [
        os.environ.get("CC", "gcc"),
        "-O2",
        "-std=c11",
        "-fPIC",
        "-shared",
        "-ffp-contract=off",
        "-fno-fast-math",
        str(INTERP_SRC),
        "-o",
        str(INTERP_SO),
        "-lm",
    ]
    subprocess.run(cmd, check=True, capture_output=True)
    return INTERP_SO


_interp_lib = None


def _lib():
    global _interp_lib
    if _interp_lib is None:
        lib = ctypes.CDLL(str(build_interp()))
        lib.li_load.restype = ctypes.c_void_p
        lib.li_load.argtypes = [ctypes.c_char_p]
        lib.li_error.restype = ctypes.c_char_p
        lib.li_run.restype = ctypes.c_int
        lib.li_run.argtypes = [
            ctypes.c_void_p,
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.c_uint64,
            ctypes.c_uint64,
            ctypes.c_void_p,
            ctypes.c_void_p,
        ]
        lib.li_free.argtypes = [ctypes.c_void_p]
        _interp_lib = lib
    return _interp_lib


def _parse_io(text: str):
    ins, outs = [], []
    for ln in text.splitlines():
        t = ln.split()
        if t and t[0] == "input":
            ins.append((t[3], t[2]))
        elif t and t[0] == "output":
            outs.append((t[3], t[2]))
    return ins, outs


class Interp:
    """The C restatement of bse for one kernel's text IR."""

    def __init__(self, name: str, ir_text: Optional[str] = None):
        self.name = name
        text = ir_text if ir_text is not None else (IR_DIR / f"{name}.lir").read_text()
        self.inputs, self.outputs = _parse_io(text)
        self._k = _lib().li_load(text.encode())
        if not self._k:
            raise ValueError(f"{name}: {_lib().li_error().decode()}")

    def __del__(self):
        k = getattr(self, "_k", None)
        if k:
            _lib().li_free(k)
            self._k = None

    def run(
        self,
        inputs: Sequence[Optional[np.ndarray]],
        n: Optional[int] = None,
        max_steps: int = 1 << 40,
        count_instr: bool = False,
        table: Optional[np.ndarray] = None,
    ):
        """Returns a list of output arrays (and per-thread instruction counts
        when ``count_instr``).  `table` holds the words of the tab op."""
        if n is None:
            n = len(next(a for a in inputs if a is not None))
        ins = [
            None if a is None else np.ascontiguousarray(a, dtype=NP_TYPE[t])
            for a, (_, t) in zip(inputs, self.inputs)
        ]
        outs = [np.zeros(n, dtype=NP_TYPE[t]) for _, t in self.outputs]
        pin = (ctypes.c_void_p * max(1, len(ins)))(
            *[None if a is None else a.ctypes.data for a in ins]
        )
        pout = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        counts = np.zeros(n, dtype=np.uint64) if count_instr else None
        tab = None if table is None else np.ascontiguousarray(table, dtype=np.uint32)
        rc = _lib().li_run(
            self._k,
            pin,
            pout,
            n,
            max_steps,
            None if counts is None else counts.ctypes.data,
            None if tab is None else tab.ctypes.data,
        )
        if rc != 0:
            raise RuntimeError(f"{self.name}: a thread exceeded max_steps")
        return (outs, counts) if count_instr else outs


# ---------------------------------------------------------------- Loom bse
_ref_lib = None


def ref_available() -> bool:
    return REF_SO.exists()


def ref_run(
    name: str,
    inputs: Sequence[Optional[np.ndarray]],
    n: int,
    threads: int = 1,
    table: Optional[np.ndarray] = None,
):
    """Run Loom's own bse (oracle/_ref/libloomref.so) on threads [0, n);
    `table` is bound for the tab op."""
    global _ref_lib
    if _ref_lib is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (oracle/build_ref.py)")
        lib = ctypes.CDLL(str(REF_SO))
        lib.loom_ref_run.restype = ctypes.c_int
        lib.loom_ref_run.argtypes = [
            ctypes.c_char_p,
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.c_uint64,
            ctypes.c_int,
            ctypes.c_void_p,
        ]
        _ref_lib = lib
    text = (IR_DIR / f"{name}.lir").read_text()
    in_decl, out_decl = _parse_io(text)
    ins = [
        None if a is None else np.ascontiguousarray(a, dtype=NP_TYPE[t])
        for a, (_, t) in zip(inputs, in_decl)
    ]
    outs = [np.zeros(n, dtype=NP_TYPE[t]) for _, t in out_decl]
    pin = (ctypes.c_void_p * max(1, len(ins)))(
        *[None if a is None else a.ctypes.data for a in ins]
    )
    pout = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
    tab = None if table is None else np.ascontiguousarray(table, dtype=np.uint32)
    rc = _ref_lib.loom_ref_run(
        name.encode(), pin, pout, n, threads, None if tab is None else tab.ctypes.data
    )
    if rc != 0:
        raise KeyError(f"{name} not in the reference runner")
    return outs


# ---------------------------------------------------------------- gang port
GANG_SO = HERE / "_lib" / "libloomgang.so"
GANG_METHODS = {"compact": 0, "hybrid": 1}
_gang_lib = None


def gang_available() -> bool:
    return GANG_SO.exists()


def gang_run(
    name: str,
    inputs: Sequence[Optional[np.ndarray]],
    n: int,
    threads: int = 1,
    table: Optional[np.ndarray] = None,
    method: str = "hybrid",
    stream: int = 288,
    utr_den: int = 16,
    stats: Optional[Dict[str, int]] = None,
):
    """Run the CPU gang port (oracle/gang_engine.hpp, Loom's compact or
    hybrid method restated) on threads [0, n) with `threads` workers, each
    with a hybrid stream of `stream` threads and utilisation threshold
    1/utr_den; a None input is the thread index.  With `stats`, fills in the
    gang block executions, the lanes active in them and the sorts."""
    global _gang_lib
    if _gang_lib is None:
        if not GANG_SO.exists():
            raise FileNotFoundError(f"{GANG_SO} not built (oracle/build_gang.py)")
        lib = ctypes.CDLL(str(GANG_SO))
        lib.loom_gang_run.restype = ctypes.c_int
        lib.loom_gang_run.argtypes = [
            ctypes.c_char_p,
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.c_uint64,
            ctypes.c_int,
            ctypes.c_void_p,
            ctypes.c_int,
            ctypes.c_uint,
            ctypes.c_uint,
            ctypes.POINTER(ctypes.c_uint64),
        ]
        _gang_lib = lib
    text = (IR_DIR / f"{name}.lir").read_text()
    in_decl, out_decl = _parse_io(text)
    ins = [None if a is None else np.ascontiguousarray(a, dtype=NP_TYPE[t]) for a, (_, t) in zip(inputs, in_decl)]
    outs = [np.zeros(n, dtype=NP_TYPE[t]) for _, t in out_decl]
    pin = (ctypes.c_void_p * max(1, len(ins)))(*[None if a is None else a.ctypes.data for a in ins])
    pout = (ctypes.c_void_p * max(1, len(outs)))(*[o.ctypes.data for o in outs])
    tab = None if table is None else np.ascontiguousarray(table, dtype=np.uint32)
    st = (ctypes.c_uint64 * 3)()
    rc = _gang_lib.loom_gang_run(
        name.encode(), pin, pout, n, threads, None if tab is None else tab.ctypes.data,
        GANG_METHODS[method], stream, utr_den, st,
    )
    if rc != 0:
        raise KeyError(f"{name} not in the gang port")
    if stats is not None:
        stats.update(blocks=int(st[0]), lanes=int(st[1]), sorts=int(st[2]))
    return outs


# ---------------------------------------------------------------- numpy refs
def val_fib(n: np.ndarray) -> np.ndarray:
    """Loom src/tests/programs.hpp:353-368: fib(n) for n <= 1 is n, else the
    iterative loop from i = 2 to n, wrapping in the integer type."""
    n = np.asarray(n)
    dt = n.dtype
    out = np.where(n <= 1, n, 0).astype(dt)
    p = np.zeros_like(n)
    c = np.ones_like(n)
    maxn = int(n.max()) if n.size else 0
    with np.errstate(over="ignore"):
        for i in range(2, maxn + 1):
            t = (p + c).astype(dt)
            live = n >= i
            p = np.where(live, c, p)
            c = np.where(live, t, c)
    return np.where(n <= 1, out, c).astype(dt)


def val_collatz(n: np.ndarray) -> np.ndarray:
    """Collatz stopping time: steps until n == 1 under n -> n/2 (even),
    3n+1 (odd); n <= 1 gives 0.  u64 arithmetic, u32 step count."""
    x = np.asarray(n, dtype=np.uint64).copy()
    steps = np.zeros(x.shape, dtype=np.uint32)
    live = x > 1
    with np.errstate(over="ignore"):
        while live.any():
            xl = x[live]
            odd = (xl & np.uint64(1)).astype(bool)
            x[live] = np.where(odd, xl * np.uint64(3) + np.uint64(1), xl >> np.uint64(1))
            steps[live] += np.uint32(1)
            live = x > 1
    return steps


def val_fac(a: np.ndarray) -> np.ndarray:
    """Loom src/tests/programs.hpp:299-305 (loom::fac, wrapping)."""
    a = np.asarray(a)
    dt = a.dtype
    out = np.ones_like(a)
    with np.errstate(over="ignore"):
        for k in range(2, int(a.max()) + 1 if a.size else 2):
            out = np.where(a >= k, (out * dt.type(k)).astype(dt), out)
    return out


def val_jmp4(i: np.ndarray) -> np.ndarray:
    """Loom src/tests/programs.hpp:325-337."""
    i = np.asarray(i)
    table = {0: 1, 1: 3, 2: 7, 3: 11}
    return np.array([table.get(int(v), int(v)) for v in i], dtype=i.dtype)


def val_inc(i: np.ndarray) -> np.ndarray:
    """Loom src/tests/programs.hpp:292-297: i + 1 in the integer type."""
    i = np.asarray(i)
    with np.errstate(over="ignore"):
        return (i + i.dtype.type(1)).astype(i.dtype)


def _uint_of(a: np.ndarray):
    return np.dtype(f"u{np.asarray(a).dtype.itemsize}")


def val_union1(i: np.ndarray) -> np.ndarray:
    """Loom src/tests/programs.hpp:307-313: the value converted to the
    unsigned integer of the float's size (truncation toward zero)."""
    i = np.asarray(i)
    return np.trunc(i).astype(_uint_of(i))


def val_union2(i: np.ndarray) -> np.ndarray:
    """Loom src/tests/programs.hpp:315-322: 200 below 0.5, else 100."""
    i = np.asarray(i)
    return np.where(i < i.dtype.type(0.5), 200, 100).astype(_uint_of(i))


def val_lshift(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Loom src/tests/programs.hpp:339-344: a << b, kept to the type."""
    a = np.asarray(a)
    return np.left_shift(a, np.asarray(b).astype(a.dtype)).astype(a.dtype)


def val_rshift(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Loom src/tests/programs.hpp:346-351: a >> b."""
    a = np.asarray(a)
    return np.right_shift(a, np.asarray(b).astype(a.dtype)).astype(a.dtype)


def val_bit_not(v: np.ndarray) -> np.ndarray:
    """Loom src/tests/programs.hpp:373-378: ~v."""
    v = np.asarray(v)
    return np.invert(v).astype(v.dtype)


# ---------------------------------------------------------------- inputs
def splitmix64(seed: int, n: int) -> np.ndarray:
    """SplitMix64 stream (Steele, Lea, Flood 2014), the documented PRNG of all
    synthetic inputs: identical arrays for the oracle and the GPU."""
    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform_int(seed: int, n: int, lo: int, hi: int) -> np.ndarray:
    """n integers uniform in [lo, hi] (inclusive), by 128-bit multiply-shift
    of SplitMix64 words (Lemire's method without rejection; bias < 2^-32
    for ranges below 2^32)."""
    z = splitmix64(seed, n)
    span = hi - lo + 1
    if span >= 1 << 63:
        return (z % np.uint64(span)) + np.uint64(lo)
    hi_bits = (z >> np.uint64(32)) * np.uint64(span)
    lo_bits = ((z & np.uint64(0xFFFFFFFF)) * np.uint64(span)) >> np.uint64(32)
    return ((hi_bits + lo_bits) >> np.uint64(32)) + np.uint64(lo)


def expand_inputs(forms, n: int, instance_starts=None, types=None):
    """Materialises input columns given as arrays or the engine's input forms
    ("iota", "local_iota", "instance", ("broadcast", value)) so the CPU
    references see exactly what the device threads read."""
    starts = None if instance_starts is None else np.asarray(instance_starts, dtype=np.uint64)
    tid = np.arange(n, dtype=np.uint64)
    inst = (
        np.zeros(n, dtype=np.uint64)
        if starts is None
        else (np.searchsorted(starts, tid, side="right") - 1).astype(np.uint64)
    )
    out = []
    for j, f in enumerate(forms):
        t = NP_TYPE[types[j]] if types else np.uint32
        if isinstance(f, np.ndarray):
            out.append(f)
        elif f == "iota" or f is None:
            out.append(tid.astype(t))
        elif f == "local_iota":
            base = np.zeros(n, dtype=np.uint64) if starts is None else starts[inst.astype(np.int64)]
            out.append((tid - base).astype(t))
        elif f == "instance":
            out.append(inst.astype(t))
        elif isinstance(f, tuple) and f[0] == "broadcast":
            out.append(np.full(n, f[1], dtype=t))
        else:
            raise ValueError(f"unknown input form {f!r}")
    return out
