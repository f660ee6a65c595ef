"""SparseMatrixCSR Product / Defect on the device through the C ABI, bit-identical
to the reference (its own outputs where the fixtures hold them, else the oracle):
csr::blocksize 1..8, FP64 / FP32, empty rows, rows of up to 200,000 entries (the
long-row path), non-square matrices whose column count is not a multiple of the
block size, and the conversion from ELL."""
import numpy as np
import pytest
import torch

import honei_b200 as hb

pytestmark = pytest.mark.gpu

from test_csr_host import CASES, oracle_case


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def upload(C):
    return hb.SparseMatrixCSR.from_arrays(C.rows, C.cols, C.Ar, C.Aj, C.Ax, blocksize=C.bs)


def run(A, x, rhs):
    dt = torch.float64 if x.dtype == np.float64 else torch.float32
    y = hb.DenseVector(A.rows(), dtype=dt)
    r = hb.DenseVector(A.rows(), dtype=dt)
    hb.Product.value(y, A, hb.DenseVector(x))
    hb.Defect.value(r, hb.DenseVector(rhs), A, hb.DenseVector(x))
    return y.numpy(), r.numpy()


@pytest.mark.parametrize("name", CASES)
def test_reference_cases(golden_csr, oracle, name):
    C = oracle_case(oracle, name)
    A = upload(C)
    Ar, Aj, Ax = A.export()
    assert golden_csr.matches(name + ".Ar", Ar) and golden_csr.matches(name + ".Aj", Aj)
    assert golden_csr.matches(name + ".Ax", Ax)
    x = oracle.uniform(C.cols, 7, C.dtype)
    rhs = oracle.uniform(C.rows, 11, C.dtype)
    y, r = run(A, x, rhs)
    assert golden_csr.matches(name + ".spmv", y)
    assert golden_csr.matches(name + ".defect", r)


def random_csr(oracle, seed, rows, cols, bs, dtype=np.float64, long_rows=(), dense_row=None):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 24, rows)
    lens[rng.integers(0, rows, rows // 13)] = 0
    idx = []
    for r in range(rows):
        if dense_row is not None and r == dense_row:
            c = np.arange(cols)
        elif r in long_rows:
            c = np.sort(rng.choice(cols, min(cols, long_rows[r]), replace=False))
        else:
            c = np.unique(rng.integers(0, cols, lens[r]))
        idx.append(c)
    indptr = np.zeros(rows + 1, np.int64)
    indptr[1:] = np.cumsum([c.size for c in idx])
    indices = np.concatenate(idx)
    vals = rng.uniform(-1, 1, indices.size).astype(dtype)
    vals[vals == 0] = dtype(0.5)
    return oracle.csr_blocked(rows, cols, indptr, indices, vals, bs)


@pytest.mark.parametrize("bs", [1, 2, 3, 8])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_skewed_rows(oracle, bs, dtype):
    rows, cols = 40000, 200003
    long_rows = {5: 3000, 777: 20000, 39999: 5000, 20000: 2049}
    C = random_csr(oracle, 17 + bs, rows, cols, bs, dtype, long_rows=long_rows, dense_row=123)
    A = upload(C)
    x = oracle.uniform(cols, 7, dtype)
    rhs = oracle.uniform(rows, 11, dtype)
    y, r = run(A, x, rhs)
    assert same_bits(y, oracle.csr_spmv(C, x))
    assert same_bits(r, oracle.csr_defect(C, rhs, x))


@pytest.mark.parametrize("L,bs", [(4, 1), (6, 2), (7, 4)])
def test_from_ell(oracle, L, bs):
    E = hb.SparseMatrixELL.poisson_q1(L)
    A = hb.SparseMatrixCSR.from_ell(E, blocksize=bs)
    C = oracle.csr_from_ell(oracle.q1_ell(L), bs)
    Ar, Aj, Ax = A.export()
    assert same_bits(Ar, C.Ar) and same_bits(Aj, C.Aj) and same_bits(Ax, C.Ax)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_q1_level10(oracle, dtype):
    """1,050,625 rows: the conversion from the device ELL and the product, against
    the oracle on the exported arrays; CSR and ELL agree where the sums coincide."""
    E = hb.SparseMatrixELL.poisson_q1(10, dtype=dtype)
    A = hb.SparseMatrixCSR.from_ell(E)
    Ar, Aj, Ax = A.export()
    C = oracle.Csr(A.rows(), A.columns(), 1, Ar, Aj, Ax)
    npdt = np.float64 if dtype == torch.float64 else np.float32
    x = oracle.uniform(A.columns(), 7, npdt)
    rhs = oracle.uniform(A.rows(), 11, npdt)
    y, r = run(A, x, rhs)
    assert same_bits(y, oracle.csr_spmv(C, x))
    assert same_bits(r, oracle.csr_defect(C, rhs, x))


def test_empty_and_sizes(oracle):
    C = oracle.csr_blocked(5, 4, np.zeros(6, np.int64), np.zeros(0, np.int64), np.zeros(0), 1)
    A = upload(C)
    y, r = run(A, np.ones(4), np.full(5, 2.0))
    assert np.array_equal(y, np.zeros(5)) and np.array_equal(r, np.full(5, 2.0))
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.Product.value(hb.DenseVector(5), A, hb.DenseVector(5))
