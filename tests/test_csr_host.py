"""SparseMatrixCSR on the CPU: the oracle's CSR construction and Product / Defect
against the reference's own outputs (tests/golden/make_csr_fixture.py), the
blocking rule against a literal restatement, and the C ABI's argument checks."""
import ctypes

import numpy as np
import pytest

from honei_b200 import _lib

CASES = ["q1_L4_bs1_f64", "q1_L4_bs2_f64", "q1_L4_bs4_f64", "q1_L6_bs1_f64", "q1_L6_bs2_f64", "q1_L6_bs4_f64",
         "q1_L6_bs1_f32", "skew_bs1_f64", "skew_bs3_f64"]


def oracle_case(oracle, name):
    dt = np.float32 if name.endswith("f32") else np.float64
    bs = int(name.split("_bs")[1].split("_")[0])
    if name.startswith("q1"):
        return oracle.csr_from_ell(oracle.q1_ell(int(name[4]), dt), bs)
    return oracle.skewed_csr(5000, 4700, bs)


@pytest.mark.parametrize("name", CASES)
def test_oracle_csr_is_the_reference(golden_csr, oracle, name):
    C = oracle_case(oracle, name)
    sc = golden_csr.scalars
    assert (C.rows, C.cols, C.bs) == (sc[name + ".rows"], sc[name + ".cols"], sc[name + ".bs"])
    assert golden_csr.matches(name + ".Ar", C.Ar)
    assert golden_csr.matches(name + ".Aj", C.Aj)
    assert golden_csr.matches(name + ".Ax", C.Ax)
    x = oracle.uniform(C.cols, 7, C.dtype)
    rhs = oracle.uniform(C.rows, 11, C.dtype)
    assert golden_csr.matches(name + ".spmv", oracle.csr_spmv(C, x))
    assert golden_csr.matches(name + ".defect", oracle.csr_defect(C, rhs, x))


def literal_create(rows_entries, bs):
    """la/sparse_matrix_csr-impl.hh:98-135 as written: a loop over each row's entries"""
    Ar, Aj, Ax = [], [], []
    gi = 0
    for cols, vals in rows_entries:
        Ar.append(gi)
        i = 0
        while i < len(cols):
            base = cols[i] - cols[i] % bs
            Aj.append(base)
            d = 0
            for b in range(bs):
                if i + d < len(cols) and base + b == cols[i + d]:
                    Ax.append(vals[i + d])
                    d += 1
                else:
                    Ax.append(0.0)
            i += d
            gi += 1
    Ar.append(gi)
    return np.array(Ar, np.uint64), np.array(Aj, np.uint64), np.array(Ax)


@pytest.mark.parametrize("bs", [1, 2, 3, 5, 8])
def test_blocking_rule(oracle, bs):
    rng = np.random.default_rng(bs)
    rows, cols = 300, 97
    entries = []
    for r in range(rows):
        k = int(rng.integers(0, 30)) if r % 7 else 0
        c = np.unique(rng.integers(0, cols, k))
        entries.append((c.tolist(), rng.uniform(0.5, 1.0, c.size).tolist()))
    indptr = np.zeros(rows + 1, np.int64)
    indptr[1:] = np.cumsum([len(c) for c, _ in entries])
    C = oracle.csr_blocked(rows, cols, indptr, np.concatenate([np.array(c, np.int64) for c, _ in entries]),
                           np.concatenate([np.array(v) for _, v in entries]), bs)
    Ar, Aj, Ax = literal_create(entries, bs)
    assert np.array_equal(C.Ar, Ar) and np.array_equal(C.Aj, Aj) and np.array_equal(C.Ax, Ax)


def test_csr_entry_points_check_arguments():
    lib = _lib.load()
    h = ctypes.c_void_p()
    u64 = lambda *v: (ctypes.c_uint64 * len(v))(*v)
    Ax = (ctypes.c_double * 4)(1, 2, 3, 4)
    ok = lambda *a: lib.hb2_csr_create(ctypes.byref(h), 0, *a)
    assert ok(2, 3, 1, u64(1, 2, 4), u64(0, 1, 2, 2), Ax, 1, None) == _lib.HB2_ERR_ARG      # Ar[0] != 0
    assert ok(2, 3, 1, u64(0, 3, 2), u64(0, 1, 2), Ax, 1, None) == _lib.HB2_ERR_ARG         # not monotone
    assert ok(2, 3, 1, u64(0, 2, 3), u64(0, 1, 3), Ax, 1, None) == _lib.HB2_ERR_ARG         # column 3 >= 3
    assert ok(2, 3, 0, u64(0, 2, 3), u64(0, 1, 2), Ax, 1, None) == _lib.HB2_ERR_ARG         # blocksize 0
    assert lib.hb2_csr_create(None, 0, 2, 3, 1, u64(0, 2, 3), u64(0, 1, 2), Ax, 1, None) == _lib.HB2_ERR_ARG
    assert lib.hb2_product_csr(None, None, None, None) == _lib.HB2_ERR_ARG
    assert lib.hb2_defect_csr(None, None, None, None, None) == _lib.HB2_ERR_ARG
    assert lib.hb2_csr_from_ell(ctypes.byref(h), None, 1, None) == _lib.HB2_ERR_ARG
