"""Seeded synthetic inputs of the workloads.

Every integer input column comes from a SplitMix64 stream (Steele, Lea,
Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014): word
i of stream `seed` is the SplitMix64 finaliser of seed + i * golden gamma,
i = 1..n.  A value uniform in [lo, hi] is the high half of the 96-bit
product of the word with the span (Lemire's multiply-shift, no rejection;
bias below 2^-32 for spans under 2^32).  The same arrays are written to the
device and given to the CPU reference.
"""

from __future__ import annotations

import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int) -> np.ndarray:
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + i * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform_int(seed: int, n: int, lo: int, hi: int) -> np.ndarray:
    """n u64 values uniform in [lo, hi] (inclusive)."""
    z = splitmix64(seed, n)
    span = hi - lo + 1
    if span >= 1 << 63:
        return (z % np.uint64(span)) + np.uint64(lo)
    with np.errstate(over="ignore"):
        hi_part = (z >> np.uint64(32)) * np.uint64(span)
        lo_part = ((z & np.uint64(0xFFFFFFFF)) * np.uint64(span)) >> np.uint64(32)
        return ((hi_part + lo_part) >> np.uint64(32)) + np.uint64(lo)
