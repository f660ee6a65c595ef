"""ctypes access to the CPU oracle (oracle/liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of bench.py
import this module, and only as the checker or the timed CPU baseline.  The
product (``honei_b200``) never imports it.  Every function mirrors the C
restatement in honei_oracle.c, which cites the reference file:line it follows.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "honei_ref")

_u64 = ctypes.c_uint64
_dbl = ctypes.c_double
_ptr = ctypes.c_void_p


def build(force: bool = False) -> str:
    """Compile honei_oracle.c into liboracle.so (no FMA contraction)."""
    src = os.path.join(HERE, "honei_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-std=c99", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
                               "-o", LIB_PATH, src, "-lm"])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        L = _lib
        L.hbo_uniform.restype = _dbl
        L.hbo_uniform.argtypes = [_u64, _u64, _dbl, _dbl]
        L.hbo_q1_m.restype = _u64
        L.hbo_q1_n.restype = _u64
        L.hbo_q1_csr_f64.restype = _u64
        L.hbo_q1_csr_f32.restype = _u64
        L.hbo_prolmat_csr_f64.restype = _u64
        L.hbo_dot_f64.restype = _dbl
        L.hbo_dot_f64.argtypes = [_u64, _ptr, _ptr]
        L.hbo_cg_q1_f64.restype = _u64
        L.hbo_cg_q1_f64.argtypes = [ctypes.c_uint, _dbl, _ptr, _ptr, _u64, _dbl]
        L.hbo_jacobi_q1_f64.argtypes = [ctypes.c_uint, _dbl, _dbl, _ptr, _ptr, _u64]
        for sfx in ("f64", "f32"):
            f = getattr(L, "hbo_mg_q1_" + sfx)
            f.restype = _u64
            f.argtypes = [ctypes.c_uint, ctypes.c_uint, _dbl, _dbl, _u64, _u64, _u64, _u64, _dbl, _dbl,
                          _ptr, _ptr, _ptr]
        for sfx in ("f64", "f32"):
            f = getattr(L, "hbo_mg_q1_cycle_" + sfx)
            f.restype = _u64
            f.argtypes = [ctypes.c_int, ctypes.c_uint, ctypes.c_uint, _dbl, _dbl, _u64, _u64, _u64, _u64, _dbl,
                          _dbl, _ptr, _ptr, _ptr]
        L.hbo_mg_ell_f64.restype = _u64
        L.hbo_mg_ell_f64.argtypes = [ctypes.c_int, ctypes.c_uint, _ptr, _ptr, _ptr, _dbl, _u64, _u64, _u64, _u64,
                                     _dbl, _dbl, _ptr, _ptr, _ptr]
        for sfx in ("f64", "f32"):
            getattr(L, "hbo_csr_spmv_" + sfx).argtypes = [_u64, _u64, _u64, _ptr, _ptr, _ptr, _ptr, _ptr]
            getattr(L, "hbo_csr_defect_" + sfx).argtypes = [_u64, _u64, _u64, _ptr, _ptr, _ptr, _ptr, _ptr, _ptr]
        for f in ("hbo_cgvar_f64", "hbo_bicgstab_f64"):
            getattr(L, f).restype = _u64
        L.hbo_cgvar_f64.argtypes = [_ptr, _ptr, _ptr, _ptr, _ptr, _u64, _dbl, ctypes.c_int]
        L.hbo_bicgstab_f64.argtypes = [_ptr, _ptr, _ptr, _ptr, _ptr, _u64, _dbl]
        for sfx in ("f64", "f32"):
            f = getattr(L, "hbo_lmg_" + sfx)
            f.restype = _u64
            f.argtypes = [ctypes.c_uint, ctypes.c_uint, _ptr, _ptr, _ptr, _ptr, _u64, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, _dbl, _u64, _dbl, _ptr]
        L.hbo_lmg_mixed.restype = _u64
        L.hbo_lmg_mixed.argtypes = [ctypes.c_uint, ctypes.c_uint, _ptr, _ptr, _ptr, _ptr, _ptr, _u64, ctypes.c_int, _dbl,
                                    _u64, _dbl, _ptr, _u64, _ptr]
        L.hbo_ir_q1.restype = _u64
        L.hbo_ir_q1.argtypes = [ctypes.c_uint, ctypes.c_uint, _dbl, _dbl, _u64, _u64, _u64, _u64, _dbl, _dbl,
                                _u64, _dbl, ctypes.c_int, _ptr, _ptr, _ptr]
        L.hbo_bf16_round.restype = _dbl
        L.hbo_bf16_round.argtypes = [_dbl]
        L.hbo_bf16_round_array.argtypes = [_u64, _ptr, _ptr]
        for sfx in ("f64", "f32"):
            getattr(L, "hbo_ell_bf16_scale_" + sfx).argtypes = [_u64, _u64, _u64, _ptr, _ptr, _ptr, ctypes.c_int, _ptr]
            getattr(L, "hbo_ell_bf16_spmv_" + sfx).argtypes = [_u64, _u64, _u64, _ptr, _ptr, _ptr, _dbl, ctypes.c_int,
                                                               _ptr, _ptr]
            getattr(L, "hbo_ell_bf16_values_" + sfx).argtypes = [_u64, _u64, _u64, _u64, _ptr, _ptr, _ptr, _dbl,
                                                                 ctypes.c_int, _ptr]
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _sfx(dtype) -> str:
    return {np.dtype(np.float64): "f64", np.dtype(np.float32): "f32"}[np.dtype(dtype)]


def q1_m(L: int) -> int:
    return (1 << L) + 1


def q1_n(L: int) -> int:
    return q1_m(L) ** 2


def uniform(n: int, seed: int, dtype=np.float64, lo=-1.0, hi=1.0) -> np.ndarray:
    out = np.empty(n, dtype=dtype)
    getattr(lib(), "hbo_uniform_fill_" + _sfx(dtype))(_p(out), _u64(n), _u64(seed), _dbl(lo), _dbl(hi))
    return out


def q1_bands(L: int, dtype=np.float64, aniso: float = 1.0) -> np.ndarray:
    """9 x n bands LL LD LU DL DD DU UL UD UU of FillMatrix<POISSON, DIRICHLET_0>."""
    n = q1_n(L)
    out = np.empty((9, n), dtype=dtype)
    getattr(lib(), "hbo_q1_bands_" + _sfx(dtype))(ctypes.c_uint(L), _dbl(aniso), _p(out))
    return out


def q1_csr(L: int, dtype=np.float64, aniso: float = 1.0):
    n = q1_n(L)
    bands = q1_bands(L, dtype, aniso)
    rp = np.empty(n + 1, np.uint64)
    ci = np.empty(9 * n, np.uint64)
    v = np.empty(9 * n, dtype)
    nnz = getattr(lib(), "hbo_q1_csr_" + _sfx(dtype))(ctypes.c_uint(L), _p(bands), _p(rp), _p(ci), _p(v))
    return rp, ci[:nnz].copy(), v[:nnz].copy()


class Ell:
    """Reference ELL arrays: Aj (uint64), Ax, Arl (uint64), stride, K, T."""

    def __init__(self, rows, cols, stride, K, T, Aj, Ax, Arl):
        self.rows, self.cols, self.stride, self.K, self.T = int(rows), int(cols), int(stride), int(K), int(T)
        self.Aj, self.Ax, self.Arl = Aj, Ax, Arl

    @property
    def dtype(self):
        return self.Ax.dtype


def ell_from_csr(rows, cols, rp, ci, v, T: int = 1) -> Ell:
    stride = _u64()
    K = _u64()
    lib().hbo_ell_dims(_u64(rows), _p(rp), _u64(T), ctypes.byref(stride), ctypes.byref(K))
    Aj = np.empty(K.value * stride.value, np.uint64)
    Ax = np.empty(K.value * stride.value, v.dtype)
    Arl = np.empty(rows, np.uint64)
    getattr(lib(), "hbo_ell_from_csr_" + _sfx(v.dtype))(
        _u64(rows), _p(rp), _p(ci), _p(v), _u64(T), stride, K, _p(Aj), _p(Ax), _p(Arl))
    return Ell(rows, cols, stride.value, K.value, T, Aj, Ax, Arl)


def q1_ell(L: int, dtype=np.float64, T: int = 1, aniso: float = 1.0) -> Ell:
    n = q1_n(L)
    rp, ci, v = q1_csr(L, dtype, aniso)
    return ell_from_csr(n, n, rp, ci, v, T)


def prolmat_csr(Lf: int):
    nf = q1_n(Lf)
    rp = np.empty(nf + 1, np.uint64)
    ci = np.empty(4 * nf, np.uint64)
    v = np.empty(4 * nf, np.float64)
    nnz = lib().hbo_prolmat_csr_f64(ctypes.c_uint(Lf), _p(rp), _p(ci), _p(v))
    return rp, ci[:nnz].copy(), v[:nnz].copy()


def transfer_ell(Lf: int, dtype=np.float64):
    """(P, R) as ELL: P = ProlongationMatrix(Lf <- Lf-1), R = Transposition(P)."""
    nf, nc = q1_n(Lf), q1_n(Lf - 1)
    rp, ci, v = prolmat_csr(Lf)
    nnz = len(ci)
    rpt = np.empty(nc + 1, np.uint64)
    cit = np.empty(nnz, np.uint64)
    vt = np.empty(nnz, np.float64)
    lib().hbo_csr_transpose_f64(_u64(nf), _u64(nc), _p(rp), _p(ci), _p(v), _p(rpt), _p(cit), _p(vt))
    P = ell_from_csr(nf, nc, rp, ci, v.astype(dtype))
    R = ell_from_csr(nc, nf, rpt, cit, vt.astype(dtype))
    return P, R


def ell_spmv(A: Ell, x: np.ndarray) -> np.ndarray:
    y = np.empty(A.rows, A.dtype)
    getattr(lib(), "hbo_ell_spmv_" + _sfx(A.dtype))(
        _u64(A.rows), _u64(A.stride), _u64(A.T), _p(A.Aj), _p(A.Ax), _p(A.Arl), _p(np.ascontiguousarray(x)), _p(y))
    return y


def ell_defect(A: Ell, rhs: np.ndarray, x: np.ndarray) -> np.ndarray:
    r = np.empty(A.rows, A.dtype)
    getattr(lib(), "hbo_ell_defect_" + _sfx(A.dtype))(
        _u64(A.rows), _u64(A.stride), _u64(A.T), _p(A.Aj), _p(A.Ax), _p(A.Arl), _p(rhs), _p(x), _p(r))
    return r


def bf16_round(t: np.ndarray) -> np.ndarray:
    """to nearest BF16 value, ties to even, from double (one rounding)"""
    t = np.ascontiguousarray(t, np.float64)
    out = np.empty_like(t)
    lib().hbo_bf16_round_array(_u64(t.size), _p(t), _p(out))
    return out


def ell_bf16_scale(A: Ell, compensate: bool):
    """(s, largest relative rounding error) of the BF16-stored copy: the first of
    s = 1, 3, ..., 15 with the smallest largest error"""
    err = np.zeros(8)
    getattr(lib(), "hbo_ell_bf16_scale_" + _sfx(A.dtype))(
        _u64(A.rows), _u64(A.stride), _u64(A.T), _p(A.Aj), _p(A.Ax), _p(A.Arl), int(compensate), _p(err))
    c = int(np.argmin(err))     # the first minimum
    return float(2 * c + 1), float(err[c])


def ell_bf16_spmv(A: Ell, s: float, compensate: bool, x: np.ndarray) -> np.ndarray:
    y = np.empty(A.rows, np.float32)
    getattr(lib(), "hbo_ell_bf16_spmv_" + _sfx(A.dtype))(
        _u64(A.rows), _u64(A.stride), _u64(A.T), _p(A.Aj), _p(A.Ax), _p(A.Arl), _dbl(s), int(compensate),
        _p(np.ascontiguousarray(x, np.float32)), _p(y))
    return y


def ell_bf16_values(A: Ell, s: float, compensate: bool) -> np.ndarray:
    out = np.empty(A.K * A.stride, np.float32)
    getattr(lib(), "hbo_ell_bf16_values_" + _sfx(A.dtype))(
        _u64(A.rows), _u64(A.stride), _u64(A.T), _u64(A.K), _p(A.Aj), _p(A.Ax), _p(A.Arl), _dbl(s), int(compensate),
        _p(out))
    return out


def ell_row_length(A: Ell) -> np.ndarray:
    Arl = np.empty(A.rows, np.uint64)
    lib().hbo_ell_row_length_f64(_u64(A.rows), _u64(A.stride), _u64(A.K), _u64(A.T), _p(A.Ax), _p(Arl))
    return Arl


def q1_spmv(bands: np.ndarray, x: np.ndarray) -> np.ndarray:
    n = bands.shape[1]
    m = int(round(n ** 0.5))
    y = np.empty(n, bands.dtype)
    getattr(lib(), "hbo_q1_spmv_" + _sfx(bands.dtype))(_u64(n), _u64(m), _p(bands), _p(x), _p(y))
    return y


def q1_defect(bands: np.ndarray, rhs: np.ndarray, x: np.ndarray) -> np.ndarray:
    n = bands.shape[1]
    m = int(round(n ** 0.5))
    r = np.empty(n, bands.dtype)
    getattr(lib(), "hbo_q1_defect_" + _sfx(bands.dtype))(_u64(n), _u64(m), _p(bands), _p(rhs), _p(x), _p(r))
    return r


def dot(x: np.ndarray, y: np.ndarray) -> float:
    if x.dtype == np.float64:
        return lib().hbo_dot_f64(_u64(len(x)), _p(x), _p(y))
    f = lib().hbo_dot_f32
    f.restype = ctypes.c_float
    return f(_u64(len(x)), _p(x), _p(y))


ALL_DIRICHLET = np.full(8, 2, np.uint64)


def prolongation(coarse: np.ndarray, n_fine: int, mask=ALL_DIRICHLET) -> np.ndarray:
    fine = np.empty(n_fine, coarse.dtype)
    mask = np.ascontiguousarray(mask, np.uint64)
    getattr(lib(), "hbo_prolongation_" + _sfx(coarse.dtype))(_u64(n_fine), _p(fine), _u64(len(coarse)),
                                                              _p(coarse), _p(mask))
    return fine


def restriction(fine: np.ndarray, n_coarse: int, mask=ALL_DIRICHLET) -> np.ndarray:
    coarse = np.empty(n_coarse, fine.dtype)
    mask = np.ascontiguousarray(mask, np.uint64)
    getattr(lib(), "hbo_restriction_" + _sfx(fine.dtype))(_u64(n_coarse), _p(coarse), _u64(len(fine)),
                                                           _p(fine), _p(mask))
    return coarse


def cg_q1(L: int, b: np.ndarray, x0=None, max_iters=2000, eps=1e-8, aniso=1.0):
    x = np.zeros(q1_n(L)) if x0 is None else np.array(x0, np.float64)
    it = lib().hbo_cg_q1_f64(L, aniso, _p(b), _p(x), max_iters, eps)
    return x, int(it)


def jacobi_q1(L: int, b: np.ndarray, x0, sweeps: int, omega=0.7, aniso=1.0):
    x = np.array(x0, np.float64)
    lib().hbo_jacobi_q1_f64(L, aniso, omega, _p(b), _p(x), sweeps)
    return x


def mg_q1(max_level: int, b: np.ndarray, x0=None, min_level=3, omega=0.7, n_pre=4, n_post=4, max_iters=100,
          max_iters_coarse=1000, eps=1e-10, coarse_eps=None, aniso=1.0, cycle="V"):
    """MG solver with V or W cycles; returns (x, used_iters, stats[4])."""
    dtype = b.dtype
    x = np.zeros(q1_n(max_level), dtype) if x0 is None else np.array(x0, dtype)
    stats = np.zeros(4)
    f = getattr(lib(), "hbo_mg_q1_cycle_" + _sfx(dtype))
    it = f({"V": 0, "W": 1}[cycle], min_level, max_level, aniso, omega, n_pre, n_post, max_iters, max_iters_coarse,
           eps, eps if coarse_eps is None else coarse_eps, _p(b), _p(x), _p(stats))
    return x, int(it), stats


class _EllView(ctypes.Structure):
    _fields_ = [("rows", _u64), ("cols", _u64), ("stride", _u64), ("K", _u64),
                ("Aj", _ptr), ("Ax", _ptr), ("Arl", _ptr)]


def _views(mats):
    arr = (_EllView * max(1, len(mats)))()
    for i, m in enumerate(mats):
        arr[i] = _EllView(m.rows, m.cols, m.stride, m.K, _p(m.Aj).value, _p(m.Ax).value, _p(m.Arl).value)
    return arr


def mg_ell(A, prol, res, b: np.ndarray, x0: np.ndarray, cycle="V", omega=0.7, n_pre=4, n_post=4, max_iters=100,
           max_iters_coarse=100, eps=1e-8, coarse_eps=None):
    """MGSolver on a hierarchy of reference ELL matrices (coarsest first; prol[i] / res[i]
    between levels i+1 and i).  Returns (x, used_iters, stats[4])."""
    x = np.array(x0, np.float64)
    stats = np.zeros(4)
    it = lib().hbo_mg_ell_f64({"V": 0, "W": 1}[cycle], len(A), _views(A), _views(prol), _views(res), omega, n_pre,
                              n_post, max_iters, max_iters_coarse, eps, eps if coarse_eps is None else coarse_eps,
                              _p(np.ascontiguousarray(b, np.float64)), _p(x), _p(stats))
    return x, int(it), stats


def ell_from_file_arrays(head, Aj, Ax) -> Ell:
    """MatrixIO<io_formats::ELL>::read_matrix (math/matrix_io.hh:466-560) on the file's
    header (size, rows, columns, stride, num_cols_per_row) and arrays; row lengths as
    the raw-array constructor computes them (la/sparse_matrix_ell-impl.hh:185-208)."""
    size, rows, cols, stride, K = (int(v) for v in head)
    E = Ell(rows, cols, stride, K, 1, np.ascontiguousarray(Aj, np.uint64), np.ascontiguousarray(Ax, np.float64),
            np.zeros(rows, np.uint64))
    E.Arl = ell_row_length(E)
    return E


def ell_transpose(A: Ell) -> Ell:
    """Transposition<Tag>::value (math/transposition.hh:36-50) followed by the
    SparseMatrixELL(SparseMatrix) constructor (la/sparse_matrix_ell-impl.hh:75-122,
    threads = 1): the nonzeros of A, each row in ascending column order, stored at
    (column, row); every result row in ascending column order; stride = rows rounded up
    to 32; num_cols_per_row = the longest row (at least 1)."""
    S = A.stride
    trows = [[] for _ in range(A.cols)]
    for r in range(A.rows):
        ent = [(int(A.Aj[r + k * S]), A.Ax[r + k * S]) for k in range(int(A.Arl[r])) if A.Ax[r + k * S] != 0]
        ent.sort(key=lambda e: e[0])
        for c, v in ent:
            trows[c].append((r, v))
    K = max([1] + [len(t) for t in trows])
    stride = 32 * ((A.cols + 31) // 32)
    Aj = np.zeros(K * stride, np.uint64)
    Ax = np.zeros(K * stride, A.Ax.dtype)
    Arl = np.zeros(A.cols, np.uint64)
    for r, t in enumerate(trows):
        Arl[r] = len(t)
        for k, (c, v) in enumerate(t):
            Aj[r + k * stride] = c
            Ax[r + k * stride] = v
    return Ell(A.cols, A.rows, stride, K, 1, Aj, Ax, Arl)


def ir_q1(max_level: int, b: np.ndarray, x0=None, min_level=3, omega=0.7, n_pre=4, n_post=4, max_inner=100,
          max_iters_coarse=1000, inner_eps=1e-3, coarse_eps=None, max_outer=100, eps=1e-10, reset_inner=False,
          aniso=1.0):
    """FP64-outer / FP32-inner-MG iterative refinement; returns (x, outer_iters, stats[4])."""
    x = np.zeros(q1_n(max_level)) if x0 is None else np.array(x0, np.float64)
    stats = np.zeros(4)
    it = lib().hbo_ir_q1(min_level, max_level, aniso, omega, n_pre, n_post, max_inner, max_iters_coarse, inner_eps,
                         inner_eps if coarse_eps is None else coarse_eps, max_outer, eps, int(reset_inner),
                         _p(b), _p(x), _p(stats))
    return x, int(it), stats


class Csr:
    """Reference SparseMatrixCSR arrays: Ar (rows + 1 block offsets), Aj (first column of
    each block), Ax (bs values per block), blocksize bs."""

    def __init__(self, rows, cols, bs, Ar, Aj, Ax):
        self.rows, self.cols, self.bs = int(rows), int(cols), int(bs)
        self.Ar = np.ascontiguousarray(Ar, np.uint64)
        self.Aj = np.ascontiguousarray(Aj, np.uint64)
        self.Ax = np.ascontiguousarray(Ax)

    @property
    def dtype(self):
        return self.Ax.dtype


def csr_blocked(rows, cols, indptr, indices, values, bs=1) -> Csr:
    """SparseMatrixCSR::Implementation::_create (la/sparse_matrix_csr-impl.hh:98-135) on
    rows given as CSR with ascending columns: consecutive entries of a row that fall in
    one aligned block of bs columns share a block; Aj = the block's first column, the
    block's bs values with zeros at the missing columns."""
    indptr = np.asarray(indptr, np.int64)
    indices = np.asarray(indices, np.int64)
    values = np.asarray(values)
    if bs == 1:
        return Csr(rows, cols, 1, indptr, indices, values.copy())
    row_of = np.repeat(np.arange(rows, dtype=np.int64), np.diff(indptr))
    blk = indices // bs
    new = np.ones(indices.size, bool)
    new[1:] = (blk[1:] != blk[:-1]) | (row_of[1:] != row_of[:-1])
    block_id = np.cumsum(new) - 1
    nblocks = int(new.sum())
    Aj = (blk[new] * bs).astype(np.uint64)
    Ax = np.zeros(nblocks * bs, values.dtype)
    Ax[block_id * bs + indices % bs] = values
    counts = np.bincount(row_of[new], minlength=rows)
    Ar = np.zeros(rows + 1, np.uint64)
    Ar[1:] = np.cumsum(counts)
    return Csr(rows, cols, bs, Ar, Aj, Ax)


def csr_from_ell(E: Ell, bs=1) -> Csr:
    """SparseMatrixCSR(SparseMatrixELL) (la/sparse_matrix_csr-impl.hh:85-96): every nonzero
    slot of the ELL arrays (la/sparse_matrix.hh:157-185), rows in ascending column order."""
    S, T = E.stride, E.T
    rows_c, rows_v = [], []
    for r in range(E.rows):
        ent = {}
        for i in range(r * T, E.K * S, S):
            for t in range(T):
                if E.Ax[i + t] != 0:
                    ent[int(E.Aj[i + t])] = E.Ax[i + t]
        cs = sorted(ent)
        rows_c.append(cs)
        rows_v.append([ent[c] for c in cs])
    indptr = np.zeros(E.rows + 1, np.int64)
    indptr[1:] = np.cumsum([len(c) for c in rows_c])
    indices = np.array([c for cs in rows_c for c in cs], np.int64)
    vals = np.array([v for vs in rows_v for v in vs], E.Ax.dtype)
    return csr_blocked(E.rows, E.cols, indptr, indices, vals, bs)


def skewed_csr(n=5000, m=4700, bs=1) -> Csr:
    """The skewed test matrix of the reference driver's csr case: empty rows (r % 11 == 3),
    one full row (n/2 + 1), rows of ~2m/3 entries (r % 500 == 7), otherwise 1..17 entries."""
    L = lib()
    u = L.hbo_uniform
    indptr, indices, vals = [0], [], []
    for r in range(n):
        ent = {}
        if r % 11 == 3:
            pass
        elif r == n // 2 + 1:
            for c in range(m):
                ent[c] = u(99, r * 10007 + c, 0.25, 1.0)
        elif r % 500 == 7:
            for c in range(m):
                if (c + r) % 3 != 2:
                    ent[c] = u(99, r * 10007 + c, -1.0, -0.25)
        else:
            for j in range(1 + (r * 7) % 17):
                c = (r + j * j * 31 + j) % m
                ent[c] = u(99, r * 10007 + c, 0.25, 1.0) * (1.0 if (r + j) % 2 else -1.0)
        cs = sorted(ent)
        indices += cs
        vals += [ent[c] for c in cs]
        indptr.append(len(indices))
    return csr_blocked(n, m, np.array(indptr), np.array(indices, np.int64), np.array(vals, np.float64), bs)


def csr_spmv(A: Csr, x: np.ndarray) -> np.ndarray:
    y = np.empty(A.rows, A.dtype)
    getattr(lib(), "hbo_csr_spmv_" + _sfx(A.dtype))(A.rows, A.bs, x.size, _p(A.Ar), _p(A.Aj), _p(A.Ax),
                                                     _p(np.ascontiguousarray(x, A.dtype)), _p(y))
    return y


def csr_defect(A: Csr, rhs: np.ndarray, x: np.ndarray) -> np.ndarray:
    r = np.empty(A.rows, A.dtype)
    getattr(lib(), "hbo_csr_defect_" + _sfx(A.dtype))(A.rows, A.bs, x.size, _p(A.Ar), _p(A.Aj), _p(A.Ax),
                                                       _p(np.ascontiguousarray(rhs, A.dtype)),
                                                       _p(np.ascontiguousarray(x, A.dtype)), _p(r))
    return r


def _precon_args(P):
    """P: a numpy vector (diagonal) or an Ell matrix"""
    if isinstance(P, np.ndarray):
        return _p(np.ascontiguousarray(P, np.float64)), None, P
    return None, _views([P]), P


def cg_var(A: Ell, P, b, x0=None, max_iters=1000, eps=1e-8, smoother=False):
    """CGSolver<Tag, methods::VAR> (or CGSmoother); returns (x, used_iters)."""
    x = np.zeros(A.rows) if x0 is None else np.array(x0, np.float64)
    pd, pv, keep = _precon_args(P)
    it = lib().hbo_cgvar_f64(_views([A]), pd, pv, _p(np.ascontiguousarray(b, np.float64)), _p(x), max_iters, eps,
                             int(smoother))
    return x, int(it)


def bicgstab(A: Ell, P, b, x0=None, max_iters=1000, eps=1e-8):
    """BiCGStabSolver<Tag, methods::VAR>; returns (x, used_iters)."""
    x = np.zeros(A.rows) if x0 is None else np.array(x0, np.float64)
    pd, pv, keep = _precon_args(P)
    it = lib().hbo_bicgstab_f64(_views([A]), pd, pv, _p(np.ascontiguousarray(b, np.float64)), _p(x), max_iters, eps)
    return x, int(it)


def jacobi_vector(A: Ell) -> np.ndarray:
    """DenseVector(n, 1) then /= A(j, j) (math/mg.hh:266-273 with damping 1)"""
    d = np.zeros(A.rows)
    S = A.stride
    for k in range(A.K):
        sl = slice(k * S, k * S + A.rows)
        hit = (A.Aj[sl] == np.arange(A.rows, dtype=np.uint64)) & (np.arange(A.rows) >= 0)
        hit &= k < A.Arl.astype(np.int64)
        d[hit] = A.Ax[sl][hit]
    return 1.0 / d


def neumann2(A: Ell) -> Ell:
    """P = 2 D^-1 - D^-1 A D^-1 on A's pattern, as the reference driver's krylov case
    builds it: p_rc = -(a_rc / (a_rr a_cc)), plus 2 / a_rr on the diagonal; rows in
    ascending column order, zeros dropped (then SparseMatrixELL(SparseMatrix))."""
    diag = 1.0 / jacobi_vector(A)
    rows_c, rows_v = [], []
    S = A.stride
    for r in range(A.rows):
        ent = {}
        for k in range(int(A.Arl[r])):
            c, a = int(A.Aj[r + k * S]), A.Ax[r + k * S]
            if a != 0:
                ent[c] = a
        cs, vs = [], []
        for c in sorted(ent):
            v = -(ent[c]) / (diag[r] * diag[c])
            if c == r:
                v += 2.0 / diag[r]
            if v != 0.0:
                cs.append(c)
                vs.append(v)
        rows_c.append(cs)
        rows_v.append(vs)
    K = max([1] + [len(c) for c in rows_c])
    stride = 32 * ((A.rows + 31) // 32)
    Aj = np.zeros(K * stride, np.uint64)
    Ax = np.zeros(K * stride)
    Arl = np.zeros(A.rows, np.uint64)
    for r in range(A.rows):
        Arl[r] = len(rows_c[r])
        for k, (c, v) in enumerate(zip(rows_c[r], rows_v[r])):
            Aj[r + k * stride] = c
            Ax[r + k * stride] = v
    return Ell(A.rows, A.cols, stride, K, 1, Aj, Ax, Arl)


def read_feast_bin(raw: bytes, dtype=np.float64):
    """math/testdata/<n>.bin of the reference: int32 n, then n doubles each of DD LL LD LU
    DL DU UL UD UU, b, the analytic solution and the reference solution.  Returns
    (bands band-major LL LD LU DL DD DU UL UD UU, b, analytic, reference) in dtype."""
    n = int(np.frombuffer(raw[:4], dtype="<i4")[0])
    v = np.frombuffer(raw[4:4 + 8 * 12 * n], dtype="<f8").reshape(12, n)
    order = [1, 2, 3, 4, 0, 5, 6, 7, 8]
    bands = np.ascontiguousarray(v[order].reshape(-1)).astype(dtype)
    return bands, v[9].astype(dtype), v[10].copy(), v[11].copy()


def lmg_dinv(bands: np.ndarray, n: int, omega=0.7) -> np.ndarray:
    """the reference tests' diags_inverted: ElementInverse(DD) in the vectors' type, then
    Scale by the double omega (the product formed in double, rounded to the type)"""
    dt = bands.dtype.type
    dd = bands[4 * n:5 * n]
    inv = np.where(dd == 0, dt(0), dt(1) / np.where(dd == 0, dt(1), dd)).astype(bands.dtype)
    return (inv.astype(np.float64) * omega).astype(bands.dtype)


def legacy_mg(bands_by_level: dict, rhs, x0, n_max_iter=16, initial_zero=True, convergence_check=False,
              is_smoother=False, tolerance=1e-8, n_pre=2, adapt=1.0, mask=ALL_DIRICHLET, dinv_by_level=None):
    """Multigrid<..., JAC, CYCLE::V, FIXED> on banded Q1 levels {level: bands}; returns (x, cycles)."""
    levels = sorted(bands_by_level)
    lmin, lmax = levels[0], levels[-1]
    dt = bands_by_level[lmax].dtype
    keep = []
    bp = (_ptr * 32)()
    dp = (_ptr * 32)()
    for l in levels:
        b = np.ascontiguousarray(bands_by_level[l], dt)
        n = b.size // 9
        d = np.ascontiguousarray(dinv_by_level[l] if dinv_by_level else lmg_dinv(b, n), dt)
        keep += [b, d]
        bp[l] = _p(b).value
        dp[l] = _p(d).value
    x = np.array(x0, dt)
    m = np.ascontiguousarray(np.asarray(mask, np.uint64))
    f = getattr(lib(), "hbo_lmg_" + _sfx(dt))
    cycles = f(lmin, lmax, bp, dp, _p(np.ascontiguousarray(rhs, dt)), _p(x), n_max_iter, int(initial_zero),
               int(convergence_check), int(is_smoother), tolerance, n_pre, adapt, _p(m))
    return x, int(cycles)


def legacy_mg_mixed(bands32_by_level: dict, bands64, b, x0, n_max_iter=2, initial_zero=True, tolerance=1e-8,
                    n_pre=2, adapt=1.0, mask=ALL_DIRICHLET, max_outer=1000):
    """Multigrid<..., MIXED>: FP32 levels {level: bands} under FP64 defect correction with
    the finest FP64 bands64 and b.  Returns (x, outer_steps, inner_cycles)."""
    levels = sorted(bands32_by_level)
    keep = []
    bp = (_ptr * 32)()
    dp = (_ptr * 32)()
    for l in levels:
        bb = np.ascontiguousarray(bands32_by_level[l], np.float32)
        d = lmg_dinv(bb, bb.size // 9)
        keep += [bb, d]
        bp[l] = _p(bb).value
        dp[l] = _p(d).value
    b64 = np.ascontiguousarray(bands64, np.float64)
    x = np.array(x0, np.float64)
    m = np.ascontiguousarray(np.asarray(mask, np.uint64))
    inner = _u64()
    outer = lib().hbo_lmg_mixed(levels[0], levels[-1], bp, dp, _p(b64), _p(np.ascontiguousarray(b, np.float64)), _p(x),
                                n_max_iter, int(initial_zero), tolerance, n_pre, adapt, _p(m), max_outer,
                                ctypes.byref(inner))
    return x, int(outer), int(inner.value)
