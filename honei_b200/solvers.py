"""HONEI's solver layer for the B200 tag: grid transfer, smoother, CG (NONE and
VAR), CGSmoother, BiCGStab, MG, the legacy banded Multigrid, IR.

Mirrors math/prolongation.hh, math/restriction.hh, math/ri.hh, math/cg.hh,
math/bicgstab.hh, math/mg.hh, math/multigrid.hh and math/ir.hh.  Each solver is one call into libhonei_b200.so; the
MG cycle runs as a captured CUDA graph.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import MgParams, NotFinite, call
from .la import DenseVector, SparseMatrixELL, _check_size, _stream, _vec, dtype_code


class methods:
    """math/methods.hh"""

    class NONE:
        pass

    class PROLMAT:
        pass

    class VAR:
        """variable preconditioning (CGSolver / BiCGStabSolver<Tag, methods::VAR>)"""
        pass


ALL_DIRICHLET = np.full(8, 2, np.uint64)


class Prolongation:
    """Prolongation<tags::B200, NONE|PROLMAT>::value(fine, coarse, mask, prolmat)."""

    @staticmethod
    def value(fine, coarse, mask=ALL_DIRICHLET, prolmat=None, method=methods.NONE, stream=None):
        fine, coarse = _vec(fine), _vec(coarse)
        if method is methods.PROLMAT:
            call("hb2_product_ell", prolmat.handle, coarse.ptr, fine.ptr, _stream(stream))
            return fine
        m = np.ascontiguousarray(mask, np.uint64)
        call("hb2_prolongation", fine.dtype, fine.ptr, fine.size(), coarse.ptr, coarse.size(),
             m.ctypes.data_as(ctypes.c_void_p), _stream(stream))
        return fine


class Restriction:
    """Restriction<tags::B200, NONE|PROLMAT>::value(coarse, fine, mask, resmat)."""

    @staticmethod
    def value(coarse, fine, mask=ALL_DIRICHLET, resmat=None, method=methods.NONE, stream=None):
        fine, coarse = _vec(fine), _vec(coarse)
        if method is methods.PROLMAT:
            call("hb2_product_ell", resmat.handle, fine.ptr, coarse.ptr, _stream(stream))
            return coarse
        m = np.ascontiguousarray(mask, np.uint64)
        call("hb2_restriction", coarse.dtype, coarse.ptr, coarse.size(), fine.ptr, fine.size(),
             m.ctypes.data_as(ctypes.c_void_p), _stream(stream))
        return coarse


class RISmoother:
    """RISmoother<tags::B200>::value(A, P, b, x, temps, max_iters) (math/ri.hh:97-133)."""

    @staticmethod
    def value(A, P, b, x, temps=None, max_iters=1, stream=None):
        P, b, x = _vec(P), _vec(b), _vec(x)
        _check_size(x.size(), A.columns())
        tmp = temps[0] if temps else DenseVector(torch.empty_like(x.elements))
        call("hb2_jacobi_ell", A.handle, P.ptr, b.ptr, x.ptr, _vec(tmp).ptr, int(max_iters), _stream(stream))
        return x

    @staticmethod
    def jacobi_precon(A, omega=0.7, stream=None) -> DenseVector:
        """PreconFill "jac": P = omega / diag(A) (math/mg.hh:266-273)."""
        P = DenseVector(A.rows(), dtype=torch.float64 if A.dtype == _lib.HB2_F64 else torch.float32)
        call("hb2_jacobi_precon", A.handle, float(omega), P.ptr, _stream(stream))
        return P


HB2_CG_VAR, HB2_BICGSTAB_VAR, HB2_CG_SMOOTHER = 0, 1, 2


class KrylovSolver:
    """A Krylov solver resident on the device (hb2_krylov): its vectors and the CUDA
    graph of a whole solve, for repeated solves with one A and P.

    method: HB2_CG_VAR (CGSolver<Tag, methods::VAR>, math/cg.hh:142-210),
    HB2_BICGSTAB_VAR (BiCGStabSolver<Tag, methods::VAR>, math/bicgstab.hh:60-210) or
    HB2_CG_SMOOTHER (CGSmoother, math/cg.hh:217-290).  P: a DenseVector (element-wise
    preconditioner) or a SparseMatrixELL."""

    def __init__(self, method, A, P, max_iters, eps_relative=1e-8, stream=None):
        if isinstance(P, SparseMatrixELL):
            pm, pd = P.handle, None
            _check_size(P.rows(), A.rows())
        else:
            P = _vec(P)
            _check_size(P.size(), A.rows())
            pm, pd = None, P.ptr
        self._keep = (A, P)
        self.method = method
        h = ctypes.c_void_p()
        call("hb2_krylov_create", ctypes.byref(h), int(method), A.handle, pm, pd, int(max_iters),
             float(eps_relative), _stream(stream))
        self._h = h
        self.n = A.rows()

    def solve(self, b, x, stream=None):
        """x = the solution from the initial guess x; returns (x, used_iters, final_defect)."""
        b, x = _vec(b), _vec(x)
        _check_size(b.size(), self.n)
        _check_size(x.size(), self.n)
        used = ctypes.c_uint64()
        defect = ctypes.c_double()
        call("hb2_krylov_solve", self._h, b.ptr, x.ptr, ctypes.byref(used), ctypes.byref(defect), _stream(stream))
        return x, used.value, defect.value

    def __del__(self):
        try:
            if self._h:
                _lib.load().hb2_krylov_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass


class CGSolver:
    """CGSolver<tags::B200, methods::NONE>::value(A, P, b, x, max_iters, used_iters, eps) (math/cg.hh:64-135);
    with method=methods.VAR, CGSolver<tags::B200, methods::VAR> (math/cg.hh:142-210), P a DenseVector
    (element-wise) or a SparseMatrixELL.

    Returns (x, used_iters, final_defect)."""

    @staticmethod
    def value(A, P, b, x, max_iters, eps_relative=1e-8, method=methods.NONE, stream=None):
        if method is methods.VAR:
            return KrylovSolver(HB2_CG_VAR, A, P, max_iters, eps_relative, stream).solve(b, x, stream)
        b, x = _vec(b), _vec(x)
        _check_size(b.size(), A.rows())
        _check_size(x.size(), A.columns())
        used = ctypes.c_uint64()
        defect = ctypes.c_double()
        call("hb2_cg_solve", A.handle, b.ptr, x.ptr, int(max_iters), float(eps_relative), ctypes.byref(used),
             ctypes.byref(defect), _stream(stream))
        return x, used.value, defect.value


class BiCGStabSolver:
    """BiCGStabSolver<tags::B200, methods::VAR>::value(A, P, b, x, max_iters, used_iters, eps)
    (math/bicgstab.hh:60-210).  Returns (x, used_iters, squared final defect)."""

    @staticmethod
    def value(A, P, b, x, max_iters, eps_relative=1e-8, stream=None):
        return KrylovSolver(HB2_BICGSTAB_VAR, A, P, max_iters, eps_relative, stream).solve(b, x, stream)


class CGSmoother:
    """CGSmoother<tags::B200>::value(A, P, b, x, temp_vecs, max_iters) (math/cg.hh:217-290):
    exactly max_iters preconditioned CG steps from x.  Returns x."""

    @staticmethod
    def value(A, P, b, x, max_iters, stream=None):
        return KrylovSolver(HB2_CG_SMOOTHER, A, P, max_iters, 0.0, stream).solve(b, x, stream)[0]


def mg_info(n_max_iter=16, initial_zero=True, convergence_check=False, is_smoother=False, tolerance=1e-8,
            n_pre_smooth=2, adapt_correction_factor=1.0, omega=0.7, macro_border_mask=None,
            adaptive=False) -> _lib.MGInfoParams:
    """MGInfo of the legacy Multigrid (math/multigrid.hh:65-149); defaults of the reference's
    banded tests (math/poisson_mg_double_banded_TEST.cc).  omega scales the inverted diagonal;
    adaptive: the MIXED class's kernel (a correction factor of 0 = alpha <d, c> / <A c, c>)."""
    mask = ALL_DIRICHLET if macro_border_mask is None else np.asarray(macro_border_mask, np.uint64)
    p = _lib.MGInfoParams(n_max_iter, int(initial_zero), int(convergence_check), int(is_smoother), tolerance,
                          n_pre_smooth, adapt_correction_factor, omega)
    for i in range(8):
        p.macro_border_mask[i] = int(mask[i])
    p.adaptive = int(adaptive)
    return p


class Multigrid:
    """Multigrid<tags::B200, tags::B200, methods::NONE, methods::JAC, methods::CYCLE::V, methods::FIXED>
    on BandedMatrixQx (math/multigrid.hh:151-466, 781-825), resident on the device.

    ``Multigrid(A, min_level, info)``: A lists the banded matrices of levels min_level ..
    max_level, coarsest first.  ``value(b, x)`` solves from x and returns (x, cycles, defect)."""

    def __init__(self, A, min_level, info: _lib.MGInfoParams | None = None, stream=None):
        self.info = info or mg_info()
        self._keep = list(A)
        arr = (ctypes.c_void_p * len(A))(*[m.handle.value for m in A])
        h = ctypes.c_void_p()
        call("hb2_lmg_create", ctypes.byref(h), int(min_level), int(min_level) + len(A) - 1, arr,
             ctypes.byref(self.info), _stream(stream))
        self._h = h
        self.n = A[-1].rows()

    def value(self, b, x, stream=None):
        b, x = _vec(b), _vec(x)
        _check_size(b.size(), self.n)
        _check_size(x.size(), self.n)
        cycles = ctypes.c_uint64()
        defect = ctypes.c_double()
        call("hb2_lmg_solve", self._h, b.ptr, x.ptr, ctypes.byref(cycles), ctypes.byref(defect), _stream(stream))
        return x, cycles.value, defect.value

    def value_mixed(self, A, b, x, max_outer=1000, stream=None):
        """Multigrid<..., MIXED>::value (math/multigrid.hh:2252-2394): this FP32 hierarchy
        under FP64 defect correction with the FP64 finest matrix A; b, x FP64.
        Returns (x, outer_steps, inner_cycles, final_defect)."""
        b, x = _vec(b), _vec(x)
        _check_size(b.size(), self.n)
        _check_size(x.size(), self.n)
        outer, inner = ctypes.c_uint64(), ctypes.c_uint64()
        defect = ctypes.c_double()
        call("hb2_lmg_solve_mixed", self._h, A.handle, b.ptr, x.ptr, int(max_outer), ctypes.byref(outer),
             ctypes.byref(inner), ctypes.byref(defect), _stream(stream))
        return x, outer.value, inner.value, defect.value

    def __del__(self):
        try:
            if self._h:
                _lib.load().hb2_lmg_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass


def mg_params(n_pre=4, n_post=4, max_iters=100, max_iters_coarse=100, eps=1e-10, coarse_eps=None, omega=0.7,
              coarse_exact=True, fused_levels=True, coarse_fp64=False, cycle="V") -> MgParams:
    """cycle: "V" (MGCycleCreation<V::STATIC>) or "W" (W::STATIC)"""
    if cycle not in ("V", "W"):
        raise ValueError("cycle must be 'V' or 'W'")
    return MgParams(n_pre, n_post, max_iters, max_iters_coarse, eps, eps if coarse_eps is None else coarse_eps,
                    omega, int(coarse_exact), int(not fused_levels), int(coarse_fp64), 1 if cycle == "W" else 0)


class MGData:
    """MGData + the V-cycle OperatorList resident on the device (math/mg.hh:57-240, 567-656).

    ``MGData.poisson_q1(min_level, max_level, ...)`` assembles the Q1 hierarchy on
    the device; ``MGData(A, prol, res, params)`` takes matrices coarsest first
    (prol[i] / res[i] connect level i and i+1)."""

    def __init__(self, A=None, prol=None, res=None, params: MgParams | None = None, stream=None, _handle=None):
        self.params = params or mg_params()
        self._keep = (A, prol, res)
        if _handle is not None:
            self._h = _handle
        else:
            n = len(A)
            arr = (ctypes.c_void_p * n)(*[m.handle.value for m in A])
            parr = (ctypes.c_void_p * max(1, n - 1))(*[m.handle.value for m in prol])
            rarr = (ctypes.c_void_p * max(1, n - 1))(*[m.handle.value for m in res])
            h = ctypes.c_void_p()
            call("hb2_mg_create", ctypes.byref(h), n, arr, parr, rarr, ctypes.byref(self.params), _stream(stream))
            self._h = h
        self.used_iters = 0
        self.used_iters_coarse = 0
        self.rnorm_initial = self.rnorm_final = float("nan")

    @classmethod
    def poisson_q1(cls, min_level, max_level, dtype=torch.float64, aniso=1.0, params: MgParams | None = None,
                   stream=None):
        params = params or mg_params()
        h = ctypes.c_void_p()
        call("hb2_mg_create_q1", ctypes.byref(h), dtype_code(dtype), min_level, max_level, float(aniso),
             ctypes.byref(params), _stream(stream))
        return cls(params=params, _handle=h)

    @classmethod
    def q1_coefficient(cls, k, min_level: int, dtype=torch.float64, params: MgParams | None = None,
                       bf16: str | None = None, stream=None):
        """The hierarchy of the variable-coefficient Q1 operator with per-cell
        coefficients k ((2^L)^2 cells, inputs.q1_coefficient_operator), rediscretised
        on the coarser levels with the cells' mean coefficients, and the Q1 grid
        transfers.  bf16 = "pure" / "compensated" (F32 only): every level above the
        coarsest stored in BF16 (SparseMatrixELL.to_bf16)."""
        from .inputs import coarsen_coefficients, q1_coefficient_operator
        npdt = np.float64 if dtype == torch.float64 else np.float32
        if bf16 not in (None, "pure", "compensated") or (bf16 and dtype != torch.float32):
            raise ValueError("bf16: None, 'pure' or 'compensated', for an F32 hierarchy")
        L = int(np.log2(k.shape[0]))
        ks = [np.asarray(k, np.float64)]
        for _ in range(L - min_level):
            ks.append(coarsen_coefficients(ks[-1]))
        ks.reverse()                                   # coarsest first
        A, P, R = [], [], []
        for i, kl in enumerate(ks):
            m = SparseMatrixELL.from_arrays(*q1_coefficient_operator(kl, npdt), stream=stream)
            if bf16 and i > 0:
                m = m.to_bf16(compensate=bf16 == "compensated", stream=stream)
            A.append(m)
            if i > 0:
                p, r = SparseMatrixELL.transfer(min_level + i, dtype, stream=stream)
                P.append(p)
                R.append(r)
        return cls(A, P, R, params=params, stream=stream)

    @property
    def handle(self):
        return self._h

    def __del__(self):
        try:
            if self._h:
                _lib.load().hb2_mg_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass


class MGSolver:
    """MGSolver<tags::B200, Norm<vnt_l_two, true>>::value(data, b, x) (math/mg.hh:1094-1127)."""

    @staticmethod
    def value(data: MGData, b, x, stream=None):
        b, x = _vec(b), _vec(x)
        stats = (ctypes.c_double * 4)()
        try:
            call("hb2_mg_solve", data.handle, b.ptr, x.ptr, stats, _stream(stream))
        finally:
            # filled also when the solve ends on a NaN defect norm (NotFinite)
            data.used_iters = int(stats[0])
            data.rnorm_initial, data.rnorm_final = stats[1], stats[2]
            data.used_iters_coarse = int(stats[3])
        return x


class IRSolver:
    """IRSolver<B200 FP64, B200 inner, Norm<l2, true>>::value (math/ir.hh:31-80).

    Returns (x, outer_iters, stats[4]): outer steps, initial and last defect norm, inner
    cycles.  A NotFinite error (NaN defect norm) carries the same list as .stats."""

    @staticmethod
    def value(A: SparseMatrixELL, b, x, inner: MGData, eps=1e-10, max_iters=100, reset_inner=False, stream=None):
        b, x = _vec(b), _vec(x)
        stats = (ctypes.c_double * 4)()
        try:
            call("hb2_ir_solve", A.handle, inner.handle, b.ptr, x.ptr, float(eps), int(max_iters),
                 int(bool(reset_inner)), stats, _stream(stream))
        except NotFinite as e:
            e.stats = list(stats)
            raise
        return x, int(stats[0]), list(stats)

    @staticmethod
    def choose_inner(A: SparseMatrixELL, b, candidates, eps=1e-10, max_iters=100, growth=0.10, reps=2,
                     stream=None):
        """Pick the inner hierarchy for repeated solves with A: solve A x = b once per
        candidate (``candidates``: name -> MGData; the first is the reference, e.g. the
        FP32-stored levels, the others e.g. BF16-stored ones), each from x = 0 with the
        inner guess reset, best of ``reps`` CUDA-event timings.  A candidate is kept
        when it converged and its inner cycles are at most (1 + growth) times the
        reference's (the BF16-matrix rule: iterations may grow by 10 % at most); the
        fastest kept one is chosen.  Returns (name, report), report[name] = {"outer",
        "inner_cycles", "ms", "kept", "converged"}."""
        b = _vec(b)
        x = DenseVector(b.size(), dtype=torch.float64)
        report, ref_cycles = {}, None
        for i, (name, inner) in enumerate(candidates.items()):
            r = {"converged": False}
            best = float("inf")
            for _ in range(reps):
                x.elements.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                try:
                    _, outer, st = IRSolver.value(A, b, x, inner, eps=eps, max_iters=max_iters, reset_inner=True,
                                                  stream=stream)
                except NotFinite as e:
                    r.update(outer=int(e.stats[0]), inner_cycles=int(e.stats[3]), error="NotFinite")
                    break
                e1.record()
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1))
                r.update(outer=outer, inner_cycles=int(st[3]), converged=st[2] <= eps * st[1])
            r["ms"] = best if r["converged"] else None
            if i == 0:
                ref_cycles = r.get("inner_cycles")
            r["kept"] = bool(r["converged"] and ref_cycles is not None and
                             r["inner_cycles"] <= (1.0 + growth) * ref_cycles)
            report[name] = r
        kept = [n for n, r in report.items() if r["kept"]]
        choice = min(kept, key=lambda n: report[n]["ms"]) if kept else next(iter(candidates))
        return choice, report


def batch_params(max_iters=100, eps=1e-8, n_pre=4, n_post=4, max_iters_coarse=100, coarse_eps=1e-10,
                 omega=0.7) -> _lib.BatchParams:
    return _lib.BatchParams(max_iters, eps, n_pre, n_post, max_iters_coarse, coarse_eps, omega)


class BatchedPoissonSolver:
    """Many Q1 Poisson systems (different levels, one or more right-hand sides
    each) solved together: CGSolver<B200, methods::VAR> (math/cg.hh:142-210)
    preconditioned by one mixed-precision MG V-cycle, every PCG step of the
    whole batch one CUDA graph.

    ``systems``: list of (level, nrhs).  Vectors are FP64 torch tensors of shape
    (nrhs, (2^level+1)^2), on the device or on the host."""

    def __init__(self, systems, coarse_level=3, params: _lib.BatchParams | None = None, stream=None):
        self.systems = [(int(l), int(k)) for l, k in systems]
        self.params = params or batch_params()
        n = len(self.systems)
        levels = (ctypes.c_uint32 * n)(*[l for l, _ in self.systems])
        nrhs = (ctypes.c_uint32 * n)(*[k for _, k in self.systems])
        h = ctypes.c_void_p()
        call("hb2_batch_create_q1", ctypes.byref(h), n, levels, nrhs, int(coarse_level), ctypes.byref(self.params),
             _stream(stream))
        self._h = h
        self.steps = 0

    @staticmethod
    def unknowns(level):
        return ((1 << level) + 1) ** 2

    def info(self):
        nv, nb, nl = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64()
        call("hb2_batch_info", self._h, ctypes.byref(nv), ctypes.byref(nb), ctypes.byref(nl))
        return {"vectors": nv.value, "device_bytes": nb.value, "launches_per_step": nl.value}

    def _buf(self, system, t):
        level, k = self.systems[system]
        if t.dtype != torch.float64 or not t.is_contiguous() or t.numel() != k * self.unknowns(level):
            raise _lib.VectorSizeDoesNotMatch(_lib.HB2_ERR_SIZE,
                                              f"system {system}: expected {k} x {self.unknowns(level)} contiguous FP64")
        return ctypes.c_void_p(t.data_ptr())

    def set_rhs(self, system, b, stream=None):
        call("hb2_batch_copy", self._h, system, 0, self._buf(system, b), _stream(stream))

    def set_guess(self, system, x, stream=None):
        call("hb2_batch_copy", self._h, system, 1, self._buf(system, x), _stream(stream))

    def solution(self, system, out=None, stream=None):
        level, k = self.systems[system]
        if out is None:
            out = torch.empty((k, self.unknowns(level)), dtype=torch.float64, device="cuda")
        call("hb2_batch_copy", self._h, system, 2, self._buf(system, out), _stream(stream))
        return out

    def start(self, system, eps=0.0, zero_guess=True, stream=None):
        call("hb2_batch_start", self._h, system, float(eps), int(bool(zero_guess)), _stream(stream))

    def step(self, steps=1, stream=None):
        """Runs `steps` PCG steps; returns the indices of the systems with nothing left to do."""
        done = (ctypes.c_uint8 * len(self.systems))()
        call("hb2_batch_step", self._h, int(steps), done, _stream(stream))
        return [i for i in range(len(self.systems)) if done[i]]

    def solve(self, zero_guess=True, stream=None):
        steps = ctypes.c_uint64()
        call("hb2_batch_solve", self._h, int(bool(zero_guess)), ctypes.byref(steps), _stream(stream))
        self.steps = steps.value
        return self.steps

    def result(self, system, rhs=0):
        """(iterations, final ||r|| / ||r0||) of one right-hand side."""
        it, rel = ctypes.c_uint64(), ctypes.c_double()
        call("hb2_batch_result", self._h, system, rhs, ctypes.byref(it), ctypes.byref(rel))
        return it.value, rel.value

    def __del__(self):
        try:
            if self._h:
                _lib.load().hb2_batch_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass
