"""Seeded input domains for every registry kernel.

The ranges restate Loom's test generators (src/tests/generators.hpp:41-206:
GM_FIB 0-80, GM_FAC 0-12/0-20, GM_U3 0-3, GM_Shift 2-10, GMFloat +-1e6,
GMFloatPositive 1e-6..1e6, GMTrig +-pi, GMCanon [0,1)) and the workload
definitions (fib n in [0, 93], Collatz n in [1, 2^32)).  Values come from
SplitMix64 (oracle.splitmix64), so the same seed gives the same arrays
everywhere.
"""

from __future__ import annotations

import math
from typing import List

import numpy as np

from oracle import oracle as O


def _floats(seed: int, n: int, lo: float, hi: float, dt) -> np.ndarray:
    z = O.splitmix64(seed, n)
    u = (z >> np.uint64(40)).astype(np.float64) * (1.0 / (1 << 24))
    return (lo + (hi - lo) * u).astype(dt)


def _ints(seed: int, n: int, lo: int, hi: int, dt) -> np.ndarray:
    return O.uniform_int(seed, n, lo, hi).astype(dt)


def _full(seed: int, n: int, dt) -> np.ndarray:
    """Every bit pattern of the type equally likely."""
    size = np.dtype(dt).itemsize
    z = O.splitmix64(seed, n) & np.uint64((1 << (8 * size)) - 1)
    return z.astype(np.dtype(f"u{size}")).view(dt)


def inputs_for(name: str, n: int, seed: int, input_types: List[str]) -> List[np.ndarray]:
    """Input columns of kernel `name` for n threads."""
    out = []
    for j, t in enumerate(input_types):
        s = seed * 7919 + j
        dt = O.NP_TYPE[t]
        if name.startswith("fib_u64"):
            a = _ints(s, n, 0, 93, dt)
        elif name.startswith("fib"):
            a = _ints(s, n, 0, 80, dt)
        elif name.startswith("collatz"):
            a = _ints(s, n, 1, (1 << 32) - 1, dt)
        elif name.startswith("fac_u32"):
            a = _ints(s, n, 0, 12, dt)
        elif name.startswith("fac"):
            a = _ints(s, n, 0, 20, dt)
        elif name.startswith("increment"):
            info = np.iinfo(dt)
            a = _full(s, n, dt)
            a = np.where(a == info.max, info.max - 1, a).astype(dt)
        elif name.startswith(("jmp4", "sct_inv", "slt_inv")):
            a = _ints(s, n, 0, 3, dt)
        elif name.startswith(("pt_const", "pt2_const", "primary_const")):
            # pixels of the square render (side in the name), encoded
            # x << 16 | y as Loom's demo does
            side = int(name.rsplit("_", 1)[1])
            xy = _ints(s, n, 0, side * side - 1, np.uint32)
            a = (((xy % side) << 16) | (xy // side)).astype(dt)
        elif name.startswith("rotl32") and j == 1:
            # rotation counts as Loom's RNG test draws them
            # (src/tests/vm_smallpt.cpp:353)
            a = _ints(s, n, 0, 31, dt)
        elif name.startswith(("lshift", "rshift")):
            a = _ints(s, n, 2, 10, dt)
        elif name.startswith("bool"):
            a = _ints(s, n, 0, 1, dt)
        elif name.startswith("bit"):
            a = _full(s, n, dt)
        elif name.startswith(("union", )):
            a = _floats(s, n, 0.0, 1.0, dt)
        elif name.startswith("sin_cos"):
            a = _floats(s, n, -math.pi, math.pi, dt)
        elif name.startswith(("sqrt", "rsqrt")):
            a = _floats(s, n, 1e-6, 1e6, dt)
        elif t in ("f32", "f64"):
            a = _floats(s, n, -1e6, 1e6, dt)
        else:
            a = _full(s, n, dt)
        out.append(np.ascontiguousarray(a, dtype=dt))
    return out
