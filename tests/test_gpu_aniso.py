"""The anisotropic Q1 variant on the device (x-coupling scaled by a factor a,
diagonal (6 + 2a) / 3; the definition is pinned in tests/test_aniso_host.py):
ELL and banded assembly, the MG solver bit for bit against the oracle -- where it
converges (a = 10) and where the reference's method diverges (a = 100) -- and the
mixed-precision IR solver."""
import numpy as np
import pytest
import torch

import honei_b200 as hb
from honei_b200 import DenseVector, SparseMatrixELL

pytestmark = pytest.mark.gpu
DEV = "cuda"


def dvec(a):
    return DenseVector(torch.from_numpy(np.ascontiguousarray(a)).to(DEV))


def host(v):
    torch.cuda.synchronize()
    return v.numpy()


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("a", [10.0, 100.0])
@pytest.mark.parametrize("L", [4, 7])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_anisotropic_assembly(oracle, L, a, dt):
    npdt = np.float64 if dt == torch.float64 else np.float32
    ref = oracle.q1_ell(L, npdt, aniso=a)
    A = SparseMatrixELL.poisson_q1(L, dt, aniso=a)
    Aj, Ax, Arl = A.export()
    assert same_bits(Aj, ref.Aj) and same_bits(Ax, ref.Ax) and same_bits(Arl, ref.Arl)
    bands = oracle.q1_bands(L, npdt, aniso=a)
    Q = hb.BandedMatrixQx.poisson_q1(L, dt, aniso=a)
    x = oracle.uniform(bands.shape[1], 7, npdt)
    for M, want in ((Q, oracle.q1_spmv(bands, x)), (A, oracle.ell_spmv(ref, x))):
        y = dvec(np.zeros(bands.shape[1], npdt))
        hb.Product.value(y, M, dvec(x))
        assert same_bits(host(y), want)


@pytest.mark.parametrize("a,cycles", [(10.0, 200), (100.0, 4)])
def test_anisotropic_mg_bit_exact(oracle, a, cycles):
    """V(4,4) with the reference-order coarse CG: the same iterates as the oracle,
    converged at a = 10; at a = 100 the same diverging iterates after 4 cycles."""
    L = 6
    A = oracle.q1_ell(L, aniso=a)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42))
    data = hb.MGData.poisson_q1(3, L, aniso=a, params=hb.mg_params(max_iters=cycles, max_iters_coarse=100, eps=1e-10,
                                                                   coarse_exact=True))
    x = dvec(np.zeros(A.rows))
    hb.MGSolver.value(data, dvec(b), x)
    xo, it, _ = oracle.mg_q1(L, b, aniso=a, max_iters=cycles, max_iters_coarse=100, eps=1e-10)
    xs = host(x)
    assert data.used_iters == it
    assert same_bits(xs, xo)
    rel = np.linalg.norm(b - oracle.ell_spmv(A, xs)) / np.linalg.norm(b)
    if a == 10.0:
        assert it < cycles and rel <= 1e-10
    else:
        assert it == cycles and rel > 1e3


def test_anisotropic_ir_mixed(oracle):
    """FP64 outer / FP32 inner MG at a = 10 reaches 1e-10 like the oracle's IR."""
    L, a = 6, 10.0
    Ao = oracle.q1_ell(L, aniso=a)
    b = oracle.ell_spmv(Ao, oracle.uniform(Ao.rows, 42))
    A = SparseMatrixELL.poisson_q1(L, aniso=a)
    inner = hb.MGData.poisson_q1(3, L, dtype=torch.float32, aniso=a,
                                 params=hb.mg_params(max_iters_coarse=1000, eps=1e-3, coarse_exact=True))
    x = dvec(np.zeros(Ao.rows))
    _, it, st = hb.IRSolver.value(A, dvec(b), x, inner, eps=1e-10)
    xs = host(x)
    assert np.linalg.norm(b - oracle.ell_spmv(Ao, xs)) < 1e-10 * st[1] * 1.001
    xr, itr, _ = oracle.ir_q1(L, b, max_iters_coarse=1000, aniso=a)
    assert abs(it - itr) <= 1
    assert np.linalg.norm(xs - xr) / np.linalg.norm(xr) < 1e-9


def test_diverging_solves_report_not_finite_with_statistics(oracle):
    """At a = 100 the defect overflows: MGSolver and IRSolver raise NotFinite and keep
    their statistics (cycles run, inner cycles)."""
    L, a = 6, 100.0
    Ao = oracle.q1_ell(L, aniso=a)
    b = dvec(oracle.ell_spmv(Ao, oracle.uniform(Ao.rows, 42)))
    data = hb.MGData.poisson_q1(3, L, aniso=a, params=hb.mg_params(max_iters=80, max_iters_coarse=100, eps=1e-10))
    x = dvec(np.zeros(Ao.rows))
    with pytest.raises(hb.NotFinite):
        hb.MGSolver.value(data, b, x)
    assert 1 <= data.used_iters <= 80
    A = SparseMatrixELL.poisson_q1(L, aniso=a)
    inner = hb.MGData.poisson_q1(3, L, dtype=torch.float32, aniso=a,
                                 params=hb.mg_params(max_iters=100, max_iters_coarse=100, eps=1e-3))
    x = dvec(np.zeros(Ao.rows))
    with pytest.raises(hb.NotFinite) as err:
        hb.IRSolver.value(A, b, x, inner, eps=1e-10, max_iters=5)
    assert len(err.value.stats) == 4 and err.value.stats[3] >= 1
