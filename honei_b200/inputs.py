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


def element_coefficients(level: int, seed: int, contrast: float = 4.0) -> np.ndarray:
    """Per-element diffusion coefficients of the (2^L)^2 cells of the level-L grid:
    contrast ** U[-1/2, 1/2) from the seeded stream, so max / min <= contrast."""
    c = 1 << level
    return np.power(contrast, uniform(c * c, seed, -0.5, 0.5)).reshape(c, c)


def coarsen_coefficients(k: np.ndarray) -> np.ndarray:
    """The coefficient of each cell of the next coarser grid: the mean of its four
    children (rediscretisation of the operator on the coarse level)."""
    return 0.25 * (k[0::2, 0::2] + k[0::2, 1::2] + k[1::2, 0::2] + k[1::2, 1::2])


def q1_coefficient_operator(k: np.ndarray, dtype=np.float64):
    """The bilinear (Q1) finite-element operator of -div(k grad u) on the unit square
    with per-cell coefficients k ((2^L)^2 cells, (2^L + 1)^2 nodes), in the layout
    of the constant-coefficient operator (math/fill_matrix.hh:37-79, k = 1 gives it:
    8/3 and -1/3): Dirichlet boundary rows are unit rows; an interior row holds its
    nine couplings in ascending column order, cell (I, J) adding k_IJ times the
    element matrix [4 -1 -2 -1; -1 4 -1 -2; -2 -1 4 -1; -1 -2 -1 4] / 6 (corners
    counter-clockwise).  Every row carries other values: no two rows repeat.

    Returns the reference ELL arrays (rows, cols, stride, num_cols_per_row, Aj, Ax,
    Arl) with stride = rows and one thread per row."""
    c = k.shape[0]
    m = c + 1
    n = m * m
    k = np.asarray(k, np.float64)
    kp = np.zeros((m + 1, m + 1))          # cells padded by one on each side
    kp[1:-1, 1:-1] = k
    # node (i, j) touches cells (i-1, j-1), (i-1, j), (i, j-1), (i, j) = kp[i, j], kp[i, j+1], kp[i+1, j], kp[i+1, j+1]
    sw, se, nw, ne = kp[:-1, :-1], kp[:-1, 1:], kp[1:, :-1], kp[1:, 1:]
    w = np.empty((9, m, m))
    w[0] = -2.0 * sw                       # (i-1, j-1)
    w[1] = -(sw + se)                      # (i-1, j)
    w[2] = -2.0 * se                       # (i-1, j+1)
    w[3] = -(sw + nw)                      # (i, j-1)
    w[4] = 4.0 * (sw + se + nw + ne)       # (i, j)
    w[5] = -(se + ne)                      # (i, j+1)
    w[6] = -2.0 * nw                       # (i+1, j-1)
    w[7] = -(nw + ne)                      # (i+1, j)
    w[8] = -2.0 * ne                       # (i+1, j+1)
    w /= 6.0
    idx = np.arange(n, dtype=np.int64).reshape(m, m)
    offs = np.array([-m - 1, -m, -m + 1, -1, 0, 1, m - 1, m, m + 1], np.int64)
    interior = np.zeros((m, m), bool)
    interior[1:-1, 1:-1] = True
    interior = interior.ravel()
    Aj = np.zeros((9, n), np.uint64)
    Ax = np.zeros((9, n), dtype)
    Arl = np.where(interior, 9, 1).astype(np.uint64)
    rows = idx.ravel()
    for s in range(9):
        Aj[s, interior] = (rows[interior] + offs[s]).astype(np.uint64)
        Ax[s, interior] = w[s].ravel()[interior].astype(dtype)
    Aj[0, ~interior] = rows[~interior].astype(np.uint64)
    Ax[0, ~interior] = 1.0
    return n, n, n, 9, Aj.ravel(), Ax.ravel(), Arl
