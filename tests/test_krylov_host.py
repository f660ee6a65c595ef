"""CGSolver VAR, BiCGStabSolver VAR and CGSmoother on the CPU: the oracle against
the reference's own results (tests/golden/make_krylov_fixture.py), and the C ABI's
argument checks."""
import ctypes

import numpy as np
import pytest

from honei_b200 import _lib


@pytest.fixture(scope="module")
def golden_kr():
    import conftest
    return conftest.Golden("reference_krylov")


def case(oracle, L):
    A = oracle.q1_ell(L)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42))
    return A, b


@pytest.mark.parametrize("L", [5, 6])
def test_preconditioners_are_the_reference(golden_kr, oracle, L):
    A, b = case(oracle, L)
    assert golden_kr.matches(f"kr_L{L}.b", b)
    P = oracle.neumann2(A)
    assert golden_kr.matches(f"kr_L{L}.Pn.Aj", P.Aj)
    assert golden_kr.matches(f"kr_L{L}.Pn.Ax", P.Ax)


@pytest.mark.parametrize("L", [5, 6])
@pytest.mark.parametrize("name", ["cgvar_jac", "cgvar_neu", "bicg_jac", "bicg_neu"])
def test_oracle_solvers_are_the_reference(golden_kr, oracle, L, name):
    A, b = case(oracle, L)
    P = oracle.jacobi_vector(A) if name.endswith("jac") else oracle.neumann2(A)
    solve = oracle.cg_var if name.startswith("cg") else oracle.bicgstab
    x, it = solve(A, P, b, max_iters=1000, eps=1e-8)
    assert it == int(golden_kr.scalar(f"kr_L{L}.{name}.iters"))
    assert golden_kr.matches(f"kr_L{L}.{name}.x", x)


@pytest.mark.parametrize("L", [5, 6])
def test_oracle_smoother_is_the_reference(golden_kr, oracle, L):
    A, b = case(oracle, L)
    x, it = oracle.cg_var(A, oracle.jacobi_vector(A), b, max_iters=5, smoother=True)
    assert it == 5
    assert golden_kr.matches(f"kr_L{L}.cgsmooth_jac.x", x)


def test_bicgstab_counts_like_the_reference(oracle):
    """used_iters = iterations + 1, and at least one iteration (a do-while)"""
    A, b = case(oracle, 5)
    P = oracle.jacobi_vector(A)
    assert oracle.bicgstab(A, P, b, max_iters=0)[1] == 2
    assert oracle.bicgstab(A, P, b, max_iters=3)[1] == 5
    assert oracle.cg_var(A, P, b, max_iters=0)[1] == 0
    assert oracle.cg_var(A, P, b, max_iters=7)[1] == 7


def test_krylov_entry_points_check_arguments():
    lib = _lib.load()
    h = ctypes.c_void_p()
    d = (ctypes.c_double * 4)()
    assert lib.hb2_krylov_create(ctypes.byref(h), 0, None, None, d, 10, 1e-8, None) == _lib.HB2_ERR_ARG
    assert lib.hb2_krylov_create(None, 0, None, None, d, 10, 1e-8, None) == _lib.HB2_ERR_ARG
    assert lib.hb2_krylov_solve(None, d, d, None, None, None) == _lib.HB2_ERR_ARG
