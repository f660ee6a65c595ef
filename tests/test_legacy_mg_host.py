"""The legacy banded Multigrid on the CPU: the oracle's restatement against the
reference's own solutions on its FEAST banded test data
(tests/golden/make_legacy_mg_fixture.py), and the C ABI's argument checks."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from honei_b200 import _lib

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_DATA = os.path.join(os.environ.get("HONEI_REFERENCE", "/nonexistent"), "honei/math/testdata/")
MIXED = [2, 1, 2, 1, 2, 2, 1, 2]
CASES = {
    "A": dict(L=5, dtype=np.float64, kw=dict(n_max_iter=16), x0=None),
    "B": dict(L=5, dtype=np.float64, kw=dict(n_max_iter=30, initial_zero=False, convergence_check=True,
                                             tolerance=1e-6, n_pre=3, adapt=0.8, mask=MIXED), x0=5),
    "C": dict(L=4, dtype=np.float64, kw=dict(n_max_iter=3, is_smoother=True), x0=None),
    "D": dict(L=5, dtype=np.float32, kw=dict(n_max_iter=16), x0=None),
}


@pytest.fixture(scope="module")
def lmg_golden():
    return dict(np.load(os.path.join(GOLDEN, "reference_legacy_mg.npz")))


def levels(golden, L, dtype):
    """{level: band-major bands (LL..UU)}, the finest b"""
    out = {}
    for l in range(1, L + 1):
        n = ((1 << l) + 1) ** 2
        v = golden[f"bin_{n}"]
        out[l] = np.ascontiguousarray(v[[1, 2, 3, 4, 0, 5, 6, 7, 8]].reshape(-1)).astype(dtype)
    n = ((1 << L) + 1) ** 2
    return out, golden[f"bin_{n}"][9].astype(dtype)


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference sources not present")
def test_fixture_is_the_reference_data(lmg_golden):
    meta = json.load(open(os.path.join(GOLDEN, "reference_legacy_mg.json")))
    for name, digest in meta["sha256"].items():
        raw = open(REF_DATA + name, "rb").read()
        assert hashlib.sha256(raw).hexdigest() == digest
        n = int(name.split(".")[0])
        assert np.array_equal(np.frombuffer(raw[4:], "<f8").reshape(12, n), lmg_golden[f"bin_{n}"])


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_is_the_reference(lmg_golden, oracle, case):
    c = CASES[case]
    bands, b = levels(lmg_golden, c["L"], c["dtype"])
    n = b.size
    x0 = oracle.uniform(n, c["x0"]) if c["x0"] else np.zeros(n)
    x, cycles = oracle.legacy_mg(bands, b, x0.astype(c["dtype"]), **c["kw"])
    ref = lmg_golden[f"lmg_{case}.x"]
    assert x.dtype == ref.dtype and np.array_equal(x.view(np.uint8), ref.view(np.uint8))


def test_reference_test_tolerance(lmg_golden):
    """the reference test's own check: within 1e-4 of the stored reference solution"""
    assert np.abs(lmg_golden["lmg_A.x"] - lmg_golden["bin_1089"][11]).max() < 1e-4


def test_lmg_entry_points_check_arguments():
    lib = _lib.load()
    h = ctypes.c_void_p()
    p = _lib.MGInfoParams()
    p.n_pre_smooth = 2
    arr = (ctypes.c_void_p * 1)()
    assert lib.hb2_lmg_create(ctypes.byref(h), 1, 2, None, ctypes.byref(p), None) == _lib.HB2_ERR_ARG
    assert lib.hb2_lmg_create(ctypes.byref(h), 0, 2, arr, ctypes.byref(p), None) == _lib.HB2_ERR_ARG
    assert lib.hb2_lmg_create(ctypes.byref(h), 3, 2, arr, ctypes.byref(p), None) == _lib.HB2_ERR_ARG
    assert lib.hb2_lmg_create(ctypes.byref(h), 1, 1, arr, None, None) == _lib.HB2_ERR_ARG
    assert lib.hb2_lmg_solve(None, None, None, None, None, None) == _lib.HB2_ERR_ARG


MIXED_CASES = {"E": dict(adapt=1.0, x0=None), "F": dict(adapt=0.0, x0=6)}


def mixed_levels(golden):
    b32, _ = levels(golden, 5, np.float32)
    b64, b = levels(golden, 5, np.float64)
    return b32, b64[5], b


@pytest.mark.parametrize("case", sorted(MIXED_CASES))
def test_oracle_mixed_is_the_reference(lmg_golden, oracle, case):
    """Multigrid<..., MIXED> in the configuration of math/poisson_mg_mixed_banded_TEST.cc"""
    c = MIXED_CASES[case]
    b32, a64, b = mixed_levels(lmg_golden)
    x0 = oracle.uniform(b.size, c["x0"]) if c["x0"] else np.zeros(b.size)
    x, outer, inner = oracle.legacy_mg_mixed(b32, a64, b, x0, adapt=c["adapt"])
    assert np.array_equal(x.view(np.uint8), lmg_golden[f"lmg_{case}.x"].view(np.uint8))
    assert inner == 2 * outer
    assert np.abs(x - lmg_golden["bin_1089"][11]).max() < 1e-4   # the reference test's check
