"""Parity at the benchmark workloads' own sizes and on the exact paths the benchmark times.

* Q1 level 10 (1,050,625 unknowns) with the benchmark's MG parameters:
  V(4,4), omega 0.7, coarse level 3, coarse CG capped at 100 iterations with
  tree-ordered dots (coarse_exact=False), stop at 1e-10.  Against the oracle
  (math/mg.hh:1094-1127 restated, reference-order coarse dots): cycle count within
  +-1, true relative residual below 1e-10 on the oracle's operator, solution within
  1e-8 relative of the oracle's.  (Each of the two solutions is about 5e-7 from the
  exact solution at this stop; the 1e-8 bound says they are the same iterate up
  to the coarse solve's rounding.)
* Q1 level 11 (4,198,401 unknowns): FP64 MG with the reference-order coarse
  solve bit for bit against the oracle; with the benchmark's coarse mode as above;
  mixed-precision IR (math/ir.hh:31-80) with its true residual below 1e-10 and its
  error stated against the oracle's FP64 MG solution, bounded by what the two
  residuals allow: ||x - x_o|| <= ||A^-1|| (||r|| + ||r_o||), with ||A^-1|| =
  1 / lambda_min of the Q1 operator (lambda_min = (8 - 4c - 4c^2) / 3,
  c = cos(pi / (m - 1)): the smoothest interior mode).
* SpMV, defect and the Jacobi sweep at level 11 on the plain layout and on the
  layout the autotuner picks: bit for bit against the oracle.
"""
import numpy as np
import pytest
import torch

import honei_b200 as hb
from honei_b200 import DenseVector, SparseMatrixELL

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-8        # benched coarse mode vs the oracle's reference-order solve


def q1_lambda_min(L):
    """smallest eigenvalue of the Q1 stencil (8/3 centre, -1/3 neighbours) on the
    interior nodes of the (2^L + 1)^2 grid with Dirichlet rows"""
    import math
    c = math.cos(math.pi / (1 << L))
    return (8.0 - 4.0 * c - 4.0 * c * c) / 3.0


def dvec(a):
    return DenseVector(torch.from_numpy(np.ascontiguousarray(a)).cuda())


def host(v):
    torch.cuda.synchronize()
    return v.numpy()


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def bench_params(eps=1e-10):
    return hb.mg_params(max_iters_coarse=100, eps=eps, coarse_exact=False)


class Case:
    def __init__(self, oracle, L):
        self.L = L
        self.A = oracle.q1_ell(L)
        self.b = oracle.ell_spmv(self.A, oracle.uniform(self.A.rows, 42))
        self.x, self.iters, _ = oracle.mg_q1(L, self.b, max_iters_coarse=100)
        self.nb = np.linalg.norm(self.b)

    def relres(self, oracle, x):
        return np.linalg.norm(self.b - oracle.ell_spmv(self.A, x)) / self.nb


@pytest.fixture(scope="module")
def case10(oracle):
    return Case(oracle, 10)


@pytest.fixture(scope="module")
def case11(oracle):
    return Case(oracle, 11)


def solve_mg(L, b, params, dtype=torch.float64):
    data = hb.MGData.poisson_q1(3, L, dtype=dtype, params=params)
    x = dvec(np.zeros(b.size))
    hb.MGSolver.value(data, dvec(b), x)
    return host(x), data.used_iters


@pytest.mark.parametrize("L", [10, 11])
def test_mg_benchmark_mode_against_the_oracle(oracle, case10, case11, L):
    c = case10 if L == 10 else case11
    x, it = solve_mg(L, c.b, bench_params())
    assert abs(it - c.iters) <= 1, (it, c.iters)
    assert c.relres(oracle, x) < 1e-10
    assert np.linalg.norm(x - c.x) / np.linalg.norm(c.x) < SOL_TOL


def test_mg_level11_reference_order_bit_exact(case11):
    x, it = solve_mg(11, case11.b, hb.mg_params(max_iters_coarse=100, eps=1e-10, coarse_exact=True))
    assert it == case11.iters
    assert same_bits(x, case11.x)


def test_mixed_ir_level11_against_the_oracle(oracle, case11):
    """The benchmark's mixed-precision IR: FP32 MG V(4,4) inner solve to 1e-3 from a
    zero start, FP64 coarse CG to the same 1e-3 (the reference's one eps for both),
    FP64 outer defect / update / norm, stop at 1e-10."""
    L = 11
    A = SparseMatrixELL.poisson_q1(L)
    inner = hb.MGData.poisson_q1(3, L, dtype=torch.float32,
                                 params=hb.mg_params(max_iters_coarse=100, eps=1e-3, coarse_eps=1e-3,
                                                     coarse_exact=False, coarse_fp64=True))
    x = dvec(np.zeros(case11.b.size))
    _, it, st = hb.IRSolver.value(A, dvec(case11.b), x, inner, eps=1e-10, reset_inner=True)
    xs = host(x)
    r_mixed, r_fp64 = case11.relres(oracle, xs), case11.relres(oracle, case11.x)
    assert r_mixed < 1e-10
    err = np.linalg.norm(xs - case11.x) / np.linalg.norm(case11.x)
    bound = (r_mixed + r_fp64) * case11.nb / (q1_lambda_min(L) * np.linalg.norm(case11.x))
    assert err < bound, (err, bound)
    assert it <= 6


@pytest.mark.parametrize("layout", ["0", None])
def test_level11_operators_bit_exact(oracle, case11, monkeypatch, layout):
    """y = A x, r = b - A x (+ ||r||^2) and one Jacobi sweep at level 11, on the plain
    layout (HB2_ELL_COMPACT=0) and on the one the autotuner picks."""
    if layout is not None:
        monkeypatch.setenv("HB2_ELL_COMPACT", layout)
    ref = case11.A
    A = SparseMatrixELL.poisson_q1(11)
    if layout == "0":
        assert A.layout()[0] == 0
    x, rhs = oracle.uniform(ref.cols, 7), oracle.uniform(ref.rows, 11)
    y = dvec(np.zeros(ref.rows))
    hb.Product.value(y, A, dvec(x))
    assert same_bits(host(y), oracle.ell_spmv(ref, x))
    r = dvec(np.zeros(ref.rows))
    nrm = torch.zeros(1, dtype=torch.float64, device="cuda")
    hb.Defect.value(r, dvec(rhs), A, dvec(x), norm2_out=nrm)
    rr = oracle.ell_defect(ref, rhs, x)
    assert same_bits(host(r), rr)
    expect = float(np.dot(rr, rr))
    assert abs(nrm.item() - expect) <= 1e-12 * expect
    P = hb.RISmoother.jacobi_precon(A, 0.7)
    x0 = x * 0.1
    xv = dvec(x0)
    hb.RISmoother.value(A, P, dvec(rhs), xv, max_iters=2)
    assert same_bits(host(xv), oracle.jacobi_q1(11, rhs, x0, 2))


@pytest.mark.parametrize("L", [7, 10])
def test_ir_graph_matches_the_host_loop(oracle, monkeypatch, L):
    """hb2_ir_solve as one CUDA graph (outer and inner loops as conditional nodes, the
    outer defect fused with its FP32 conversion) against the same solve with the loop
    on the host (HB2_IR_LOOP=host): the same outer and inner step counts, the same
    solution (bit for bit where both reduce the outer norm in the same order)."""
    A0 = oracle.q1_ell(L)
    b = oracle.ell_spmv(A0, oracle.uniform(A0.rows, 42))
    A = SparseMatrixELL.poisson_q1(L)
    out = []
    for mode in (None, "host"):
        if mode:
            monkeypatch.setenv("HB2_IR_LOOP", mode)
        inner = hb.MGData.poisson_q1(3, L, dtype=torch.float32,
                                     params=hb.mg_params(max_iters_coarse=100, eps=1e-3, coarse_eps=1e-3,
                                                         coarse_exact=False, coarse_fp64=True))
        x = dvec(np.zeros(A0.rows))
        _, it, st = hb.IRSolver.value(A, dvec(b), x, inner, eps=1e-10, reset_inner=True)
        out.append((host(x), it, st))
    (xg, itg, stg), (xh, ith, sth) = out
    assert itg == ith and stg[3] == sth[3]
    assert np.linalg.norm(xg - xh) <= 1e-13 * np.linalg.norm(xh)
    assert abs(stg[2] - sth[2]) <= 1e-10 * sth[2]
    assert np.linalg.norm(b - oracle.ell_spmv(A0, xg)) < 1e-10 * np.linalg.norm(b) * 1.001


@pytest.mark.parametrize("L", [9, 11])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_fused_convergence_norm(oracle, monkeypatch, L, dt):
    """The MG loop with its convergence norm ||b - A x|| taken from the next cycle's
    first finest-level sweep (HB2_MG_FUSED_NORM=1) against a separate defect pass per
    cycle (the default); on the device loop and on the host loop (HB2_MG_LOOP=host):
    the same cycles, the same solution bits, the final norms within 1e-12 relative, and
    in the reference-order mode the oracle's iterates bit for bit."""
    npdt = np.float64 if dt == torch.float64 else np.float32
    A = oracle.q1_ell(L, npdt)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42, npdt))
    eps = 1e-10 if dt == torch.float64 else 1e-5
    out = {}
    for fused in ("1", "0"):
        for loop in (None, "host"):
            monkeypatch.setenv("HB2_MG_FUSED_NORM", fused)
            if loop:
                monkeypatch.setenv("HB2_MG_LOOP", loop)
            else:
                monkeypatch.delenv("HB2_MG_LOOP", raising=False)
            data = hb.MGData.poisson_q1(3, L, dtype=dt,
                                        params=hb.mg_params(max_iters_coarse=100, eps=eps, coarse_exact=True))
            x = dvec(np.zeros(A.rows, npdt))
            hb.MGSolver.value(data, dvec(b), x)
            out[(fused, loop)] = (host(x), data.used_iters, data.rnorm_final)
    ref = out[("0", None)]
    for key, (x, it, rn) in out.items():
        assert it == ref[1], key
        assert same_bits(x, ref[0]), key
        assert abs(rn - ref[2]) <= 1e-12 * ref[2], key
    if L == 9:
        xo, ito, _ = oracle.mg_q1(L, b, max_iters_coarse=100, eps=eps)
        assert ref[1] == ito and same_bits(ref[0], xo)


def test_fused_norm_stops_at_the_cycle_cap(monkeypatch):
    """max_iters cycles: the loop runs exactly that many, with or without the fused norm"""
    L = 9
    n = ((1 << L) + 1) ** 2
    b = DenseVector(torch.rand(n, dtype=torch.float64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(7)))
    res = []
    for fused in ("1", "0"):
        monkeypatch.setenv("HB2_MG_FUSED_NORM", fused)
        data = hb.MGData.poisson_q1(3, L, params=hb.mg_params(max_iters=3, max_iters_coarse=100, eps=1e-14))
        x = DenseVector(torch.zeros(n, dtype=torch.float64, device="cuda"))
        hb.MGSolver.value(data, b, x)
        res.append((host(x), data.used_iters, data.rnorm_final))
    assert res[0][1] == res[1][1] == 3
    assert same_bits(res[0][0], res[1][0])
    assert abs(res[0][2] - res[1][2]) <= 1e-12 * res[1][2]
