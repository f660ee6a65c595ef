"""The CPU oracle (oracle/honei_oracle.c) pinned bit-for-bit against fixtures that the
reference's own tags::CPU code produced (tests/golden/make_golden.py)."""
import numpy as np
import pytest


def ell_ok(golden, name, A):
    return (golden.matches(name + ".Aj", A.Aj) and golden.matches(name + ".Ax", A.Ax)
            and golden.matches(name + ".Arl", A.Arl)
            and golden.scalar(name + ".stride") == A.stride and golden.scalar(name + ".K") == A.K
            and golden.scalar(name + ".rows") == A.rows and golden.scalar(name + ".T") == A.T)


@pytest.mark.parametrize("L", range(1, 9))
def test_q1_ell_assembly_f64(golden, oracle, L):
    """FillMatrix<POISSON, DIRICHLET_0> -> SparseMatrix -> SparseMatrixELL, bit-exact."""
    A = oracle.q1_ell(L)
    assert ell_ok(golden, f"ell_L{L}_T1_f64", A)


@pytest.mark.parametrize("L", range(1, 7))
def test_q1_ell_assembly_f32(golden, oracle, L):
    A = oracle.q1_ell(L, np.float32)
    assert ell_ok(golden, f"ell_L{L}_T1_f32", A)


@pytest.mark.parametrize("T", [2, 3])
@pytest.mark.parametrize("L", [2, 3, 4])
def test_ell_threads_layout(golden, oracle, L, T):
    """ell::threads > 1: slot k of row r at (k%T) + r*T + (k/T)*stride."""
    A = oracle.q1_ell(L, T=T)
    assert ell_ok(golden, f"ell_L{L}_T{T}_f64", A)
    y = oracle.ell_spmv(A, oracle.uniform(A.cols, 7))
    assert golden.matches(f"spmv_L{L}_T{T}_f64", y)


@pytest.mark.parametrize("L", range(2, 9))
def test_transfer_matrices(golden, oracle, L):
    """ProlongationMatrix + Transposition as ELL, bit-exact."""
    P, R = oracle.transfer_ell(L)
    assert ell_ok(golden, f"prol_L{L}_f64", P)
    assert ell_ok(golden, f"res_L{L}_f64", R)


def test_row_length_matches_constructor(oracle):
    """The raw-array constructor's row_length() reproduces the assembled Arl."""
    for L in (2, 4, 6):
        A = oracle.q1_ell(L)
        assert np.array_equal(oracle.ell_row_length(A), A.Arl)


@pytest.mark.parametrize("L", range(1, 8))
def test_spmv_defect(golden, oracle, L):
    A = oracle.q1_ell(L)
    x, rhs = oracle.uniform(A.cols, 7), oracle.uniform(A.rows, 11)
    assert golden.matches(f"spmv_L{L}_f64", oracle.ell_spmv(A, x))
    assert golden.matches(f"defect_L{L}_f64", oracle.ell_defect(A, rhs, x))
    Af = oracle.q1_ell(L, np.float32)
    xf, rf = oracle.uniform(A.cols, 7, np.float32), oracle.uniform(A.rows, 11, np.float32)
    assert golden.matches(f"spmv_L{L}_f32", oracle.ell_spmv(Af, xf))
    assert golden.matches(f"defect_L{L}_f32", oracle.ell_defect(Af, rf, xf))
    B = oracle.q1_bands(L)
    assert golden.matches(f"q1spmv_L{L}_f64", oracle.q1_spmv(B, x))
    assert golden.matches(f"q1defect_L{L}_f64", oracle.q1_defect(B, rhs, x))


@pytest.mark.parametrize("L", range(2, 8))
def test_grid_transfer_ops(golden, oracle, L):
    nf, nc = oracle.q1_n(L), oracle.q1_n(L - 1)
    c, f = oracle.uniform(nc, 31), oracle.uniform(nf, 32)
    P, R = oracle.transfer_ell(L)
    assert golden.matches(f"prolong_L{L}_f64", oracle.prolongation(c, nf))
    assert golden.matches(f"restrict_L{L}_f64", oracle.restriction(f, nc))
    assert golden.matches(f"prolmat_L{L}_f64", oracle.ell_spmv(P, c))
    assert golden.matches(f"resmat_L{L}_f64", oracle.ell_spmv(R, f))


def test_blas1(golden, oracle):
    a, b = oracle.uniform(1000, 21), oracle.uniform(1000, 22)
    assert oracle.dot(a, b) == golden.scalar("dot_1000_f64")
    assert oracle.dot(a, a) == golden.scalar("norm2sq_1000_f64")
    assert np.sqrt(oracle.dot(a, a)) == golden.scalar("norm2_1000_f64")
    # element-wise updates round the product and the sum separately
    assert golden.matches("scaledsum2_1000_f64", a + 0.375 * b)
    assert golden.matches("scaledsum3_1000_f64", -1.25 * b + a)


@pytest.mark.parametrize("L", [3, 4, 5, 6])
def test_jacobi(golden, oracle, L):
    b = oracle.uniform(oracle.q1_n(L), 5)
    x = oracle.jacobi_q1(L, b, np.zeros_like(b), 4)
    assert golden.matches(f"jacobi_L{L}_f64", x)


@pytest.mark.parametrize("L", [5, 7])
def test_cg(golden, oracle, L):
    """The CPU-sized CG workload: plain CG, b = A u*, x0 = 0, rel. tol 1e-8; iterates bit-identical."""
    A = oracle.q1_ell(L)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42))
    assert golden.matches(f"cg_L{L}.b", b)
    x, it = oracle.cg_q1(L, b)
    assert it == golden.scalar(f"cg_L{L}.iters")
    assert golden.matches(f"cg_L{L}.x", x)


@pytest.mark.parametrize("L", [5, 6, 7])
def test_mg(golden, oracle, L):
    """MG V(4,4), Jacobi 0.7, coarse CG on level 3 (1000 iterations cap), eps 1e-10."""
    A = oracle.q1_ell(L)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42))
    x, it, st = oracle.mg_q1(L, b, max_iters_coarse=1000)
    assert it == golden.scalar(f"mg_L{L}.iters")
    assert st[3] == golden.scalar(f"mg_L{L}.coarse_iters")
    assert golden.matches(f"mg_L{L}.x", x)


def test_mg_f32(golden, oracle):
    A = oracle.q1_ell(6, np.float32)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42, np.float32))
    x, it, _ = oracle.mg_q1(6, b, eps=1e-5, max_iters_coarse=1000)
    assert it == golden.scalar("mg32_L6.iters")
    assert golden.matches("mg32_L6.x", x)


@pytest.mark.parametrize("L", [5, 6])
def test_ir(golden, oracle, L):
    """IRSolver: FP64 outer, FP32 inner MG with eps 1e-3 (inner guess carried over)."""
    A = oracle.q1_ell(L)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42))
    x, it, _ = oracle.ir_q1(L, b, max_iters_coarse=1000)
    assert it == golden.scalar(f"ir_L{L}.iters")
    assert golden.matches(f"ir_L{L}.x", x)


def test_coarse_cap_does_not_change_mg_convergence(oracle):
    """The coarse CG on the non-symmetric Dirichlet-row operator stagnates near 4e-7,
    so it always runs to its cap; the MG cycle count does not depend on the cap."""
    A = oracle.q1_ell(6)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42))
    its = {cap: oracle.mg_q1(6, b, max_iters_coarse=cap)[1] for cap in (20, 100, 1000)}
    assert len(set(its.values())) == 1
