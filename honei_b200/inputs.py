"""Seeded synthetic inputs: u* ~ U[lo, hi) from the splitmix64 stream (Steele, Lea,
Flood 2014), element i = mix(seed + (i+1) * golden_gamma).  Counter-based, so any
slice can be produced independently; identical to the oracle's generator."""
from __future__ import annotations

import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def uniform(n: int, seed: int, lo: float = -1.0, hi: float = 1.0, dtype=np.float64) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (np.arange(1, n + 1, dtype=np.uint64) * _GAMMA)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return (lo + (hi - lo) * u).astype(dtype)
