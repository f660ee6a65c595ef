"""The anisotropic Q1 variant on the CPU oracle: the operator's definition and the
stability of the reference's MG method on it.

The reference has no anisotropic generator.  This build's variant scales the
x-coupling (bands DL and DU, the left and right neighbours in a grid row) of the
Q1 stencil by a factor a and raises the diagonal to (6 + 2a) / 3, so interior row
sums stay zero; Dirichlet rows stay identity rows.  The MG method of the headline
workloads (V(4,4), damped Jacobi omega 0.7, rediscretised coarse operators, coarse
CG) converges on it up to a factor of about 10 and diverges from about 20: at
100, the factor of the mixed-precision stability probe, the defect grows by orders
of magnitude per cycle even without a coarse solve."""
import numpy as np
import pytest


@pytest.mark.parametrize("a", [1.0, 10.0, 100.0])
def test_anisotropic_operator_definition(oracle, a):
    L = 4
    A = oracle.q1_ell(L, aniso=a)
    m = (1 << L) + 1
    dense = np.zeros((A.rows, A.cols))
    for k in range(A.K):
        for r in range(A.rows):
            if k < A.Arl[r]:
                dense[r, int(A.Aj[k * A.stride + r])] += A.Ax[k * A.stride + r]
    interior = [r for r in range(A.rows) if 0 < r // m < m - 1 and 0 < r % m < m - 1]
    for r in interior:
        assert dense[r, r] == (8.0 / 3.0 if a == 1.0 else (6.0 + 2.0 * a) / 3.0)
        assert dense[r, r - 1] == dense[r, r + 1] == (-1.0 / 3.0 if a == 1.0 else -a / 3.0)
        assert dense[r, r - m] == dense[r, r + m] == -1.0 / 3.0
        assert abs(dense[r].sum()) < 1e-12 * a
    boundary = [r for r in range(A.rows) if r not in set(interior)]
    for r in boundary:
        assert dense[r, r] == 1.0 and np.count_nonzero(dense[r]) == 1


def _relres(oracle, L, a, cycles, cap=100):
    n = oracle.q1_n(L)
    A = oracle.q1_ell(L, aniso=a)
    b = oracle.ell_spmv(A, oracle.uniform(n, 42))
    x, it, _ = oracle.mg_q1(L, b, aniso=a, max_iters=cycles, max_iters_coarse=cap, eps=1e-10)
    return it, np.linalg.norm(b - oracle.ell_spmv(A, x)) / np.linalg.norm(b)


def test_reference_method_converges_at_factor_10(oracle):
    it, rel = _relres(oracle, 5, 10.0, 200)
    assert it < 60 and rel <= 1e-10


@pytest.mark.parametrize("cap", [0, 100])
def test_reference_method_diverges_at_factor_100(oracle, cap):
    """With or without the coarse solve the cycle amplifies the defect: the
    instability is the smoother / rediscretised coarse-grid pair, not the coarse CG."""
    _, rel1 = _relres(oracle, 6, 100.0, 1, cap)
    _, rel5 = _relres(oracle, 6, 100.0, 5, cap)
    assert rel5 > 1.0 and rel5 > 100.0 * rel1
