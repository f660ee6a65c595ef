"""CGSolver VAR, BiCGStabSolver VAR and CGSmoother on the device through the C ABI,
against the reference's results (tests/golden/make_krylov_fixture.py) and the
oracle.  The device reduces dot products in a fixed tree order where the reference
sums sequentially, so iteration counts may differ by one; the reference's own
stopping criterion must hold for the device's result."""
import numpy as np
import pytest
import torch

import honei_b200 as hb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden_kr():
    import conftest
    return conftest.Golden("reference_krylov")


def problem(oracle, L, pname):
    A = oracle.q1_ell(L)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42))
    P = oracle.jacobi_vector(A) if pname == "jac" else oracle.neumann2(A)
    dA = hb.SparseMatrixELL.from_arrays(A.rows, A.cols, A.stride, A.K, A.Aj, A.Ax, A.Arl)
    dP = hb.DenseVector(P) if pname == "jac" else hb.SparseMatrixELL.from_arrays(P.rows, P.cols, P.stride, P.K, P.Aj,
                                                                                  P.Ax, P.Arl)
    return A, P, b, dA, dP


def relres(oracle, A, b, x):
    r = oracle.ell_defect(A, b, x)
    return np.sqrt(np.dot(r, r)) / np.sqrt(np.dot(b, b))


@pytest.mark.parametrize("L", [5, 6])
@pytest.mark.parametrize("pname", ["jac", "neu"])
def test_cg_var(golden_kr, oracle, L, pname):
    A, P, b, dA, dP = problem(oracle, L, pname)
    x, used, defect = hb.CGSolver.value(dA, dP, hb.DenseVector(b), hb.DenseVector(A.rows), 1000, 1e-8,
                                        method=hb.methods.VAR)
    ref_it = int(golden_kr.scalar(f"kr_L{L}.cgvar_{pname}.iters"))
    assert abs(used - ref_it) <= 1
    assert relres(oracle, A, b, x.numpy()) < 1.05e-8      # ||r|| < eps ||r0||, x0 = 0
    xo, _ = oracle.cg_var(A, P, b)
    assert np.abs(x.numpy() - xo).max() < 1e-6 * np.abs(xo).max()


@pytest.mark.parametrize("L", [5, 6])
@pytest.mark.parametrize("pname", ["jac", "neu"])
def test_bicgstab(golden_kr, oracle, L, pname):
    A, P, b, dA, dP = problem(oracle, L, pname)
    x, used, defect = hb.BiCGStabSolver.value(dA, dP, hb.DenseVector(b), hb.DenseVector(A.rows), 1000, 1e-8)
    ref_it = int(golden_kr.scalar(f"kr_L{L}.bicg_{pname}.iters"))
    assert abs(used - ref_it) <= 1
    # squared norms against eps: ||r|| < sqrt(eps) ||r0||
    assert defect < 1e-8 * np.dot(b, b)
    assert relres(oracle, A, b, x.numpy()) < 1.05e-4
    xo, _ = oracle.bicgstab(A, P, b)
    assert np.abs(x.numpy() - xo).max() < 1e-3 * np.abs(xo).max()


@pytest.mark.parametrize("L", [5, 6])
def test_cg_smoother(golden_kr, oracle, L):
    A, P, b, dA, dP = problem(oracle, L, "jac")
    x = hb.CGSmoother.value(dA, dP, hb.DenseVector(b), hb.DenseVector(A.rows), 5)
    xr = golden_kr.array(f"kr_L{L}.cgsmooth_jac.x") if golden_kr.full.get(f"kr_L{L}.cgsmooth_jac.x") is not None \
        else oracle.cg_var(A, P, b, max_iters=5, smoother=True)[0]
    assert np.allclose(x.numpy(), xr, rtol=1e-10, atol=1e-12 * np.abs(xr).max())


@pytest.mark.parametrize("max_iters", [0, 1, 3, 10])
def test_iteration_caps(oracle, max_iters):
    A, P, b, dA, dP = problem(oracle, 5, "jac")
    _, used, _ = hb.CGSolver.value(dA, dP, hb.DenseVector(b), hb.DenseVector(A.rows), max_iters, 1e-8,
                                   method=hb.methods.VAR)
    assert used == oracle.cg_var(A, P, b, max_iters=max_iters)[1]
    _, used, _ = hb.BiCGStabSolver.value(dA, dP, hb.DenseVector(b), hb.DenseVector(A.rows), max_iters, 1e-8)
    assert used == oracle.bicgstab(A, P, b, max_iters=max_iters)[1]


def test_handle_reuse_is_deterministic(oracle):
    A, P, b, dA, dP = problem(oracle, 6, "neu")
    for method in (hb.HB2_CG_VAR, hb.HB2_BICGSTAB_VAR):
        K = hb.KrylovSolver(method, dA, dP, 1000, 1e-8)
        x1, u1, d1 = K.solve(hb.DenseVector(b), hb.DenseVector(A.rows))
        x2, u2, d2 = K.solve(hb.DenseVector(b), hb.DenseVector(A.rows))
        assert u1 == u2 and d1 == d2 and np.array_equal(x1.numpy(), x2.numpy())


@pytest.mark.parametrize("method", ["cg", "bicg"])
def test_level8(oracle, method):
    A, P, b, dA, dP = problem(oracle, 8, "neu")
    if method == "cg":
        x, used, _ = hb.CGSolver.value(dA, dP, hb.DenseVector(b), hb.DenseVector(A.rows), 2000, 1e-8,
                                       method=hb.methods.VAR)
        xo, ito = oracle.cg_var(A, P, b, max_iters=2000)
        assert relres(oracle, A, b, x.numpy()) < 1.05e-8
    else:
        x, used, _ = hb.BiCGStabSolver.value(dA, dP, hb.DenseVector(b), hb.DenseVector(A.rows), 2000, 1e-8)
        xo, ito = oracle.bicgstab(A, P, b, max_iters=2000)
        assert relres(oracle, A, b, x.numpy()) < 1.05e-4
    assert abs(used - ito) <= max(1, ito // 50)
