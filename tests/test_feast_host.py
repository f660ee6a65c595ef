"""MatrixIO / VectorIO formats, Transposition and the W-cycle on the reference's own
FEAST test data (math/testdata/poisson, read by math/mg_TEST.cc:398-463), checked
on the CPU: the oracle against the reference's results, the file readers' parsing
rules, and the C ABI's argument checks for the file entry points."""
import ctypes
import hashlib
import os

import numpy as np
import pytest

from honei_b200 import _lib
from honei_b200.io import parse_exp

REF_DATA = os.path.join(os.environ.get("HONEI_REFERENCE", "/nonexistent"), "honei/math/testdata/poisson/")


def test_parse_exp_rules():
    # VectorIO<EXP>::read_vector (math/vector_io.hh:55-110): '#' lines skipped,
    # leading blanks ignored, an unterminated last line dropped
    text = "# header\n1.5\n  -2e-3\n# 7\n3\n4"
    assert parse_exp(text).tolist() == [1.5, -2e-3, 3.0]
    assert parse_exp("").size == 0
    assert parse_exp("5\n").tolist() == [5.0]


def test_fixture_shapes(feast):
    z = feast.z
    for i in range(1, 7):
        size, rows, cols, stride, K = feast.head(f"A_{i}")
        assert rows == cols == (2 ** i + 1) ** 2 and size == stride * K and stride % 32 == 0
        assert z[f"A_{i}.Aj"].size == z[f"A_{i}.Ax"].size == size
    for i in range(2, 7):
        _, rows, cols, _, _ = feast.head(f"prol_{i}")
        assert (rows, cols) == ((2 ** i + 1) ** 2, (2 ** (i - 1) + 1) ** 2)
        assert feast.head(f"res_{i}")[1:3] == [cols, rows]
    n = (2 ** 6 + 1) ** 2
    for name in ("rhs_6", "init_6", "sol_6", "ref_x"):
        assert z[name].shape == (n,)
    assert feast.meta["used_iters"] == 8 and feast.meta["used_iters_coarse"] == 1


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference sources not present")
def test_fixture_is_the_reference_data(feast):
    for name, digest in feast.meta["sha256"].items():
        data = open(REF_DATA + name, "rb").read()
        if name.endswith(".ell"):
            assert feast.file_bytes(name[:-4]) == data
        else:
            assert hashlib.sha256(data).hexdigest() == digest
            assert np.array_equal(parse_exp(data.decode()), feast.z[name])


def test_oracle_transpose_is_the_reference_restriction(feast, oracle):
    for i in range(2, 7):
        R = oracle.ell_transpose(feast.ell(oracle, f"prol_{i}"))
        assert [R.K * R.stride, R.rows, R.cols, R.stride, R.K] == feast.head(f"res_{i}")
        assert np.array_equal(R.Aj, feast.z[f"res_{i}.Aj"].astype(np.uint64))
        assert np.array_equal(R.Ax.view(np.uint64), feast.z[f"res_{i}.Ax"].view(np.uint64))


def feast_hierarchy(feast, oracle):
    A = [feast.ell(oracle, f"A_{i}") for i in range(1, 7)]
    P = [feast.ell(oracle, f"prol_{i}") for i in range(2, 7)]
    R = [feast.ell(oracle, f"res_{i}") for i in range(2, 7)]
    return A, P, R


def test_oracle_w_cycle_is_the_reference_solve(feast, oracle):
    """MGSolverTestQuad: W-cycle, V(4,4) Jacobi 0.7, coarse CG on level 1, eps 1e-8,
    100 / 100 iteration caps -- bit-identical solution and iteration counts."""
    A, P, R = feast_hierarchy(feast, oracle)
    x, it, stats = oracle.mg_ell(A, P, R, feast.z["rhs_6"], feast.z["init_6"], cycle="W", eps=1e-8)
    assert it == feast.meta["used_iters"] and int(stats[3]) == feast.meta["used_iters_coarse"]
    assert np.array_equal(x.view(np.uint64), feast.z["ref_x"].view(np.uint64))
    # the reference test's own acceptance: within 8e-3 of sol_6
    assert np.abs(x - feast.z["sol_6"]).max() < 8e-3


def test_oracle_v_and_w_cycles_differ(feast, oracle):
    A, P, R = feast_hierarchy(feast, oracle)
    xv, itv, _ = oracle.mg_ell(A, P, R, feast.z["rhs_6"], feast.z["init_6"], cycle="V", eps=1e-8)
    assert itv > feast.meta["used_iters"]
    assert np.abs(xv - feast.z["sol_6"]).max() < 8e-3


def test_oracle_q1_w_cycle_converges(oracle):
    L = 6
    n = oracle.q1_n(L)
    b = oracle.uniform(n, 11)
    xv, itv, sv = oracle.mg_q1(L, b, min_level=2, eps=1e-10, cycle="V")
    xw, itw, sw = oracle.mg_q1(L, b, min_level=2, eps=1e-10, cycle="W")
    assert sw[2] < 1e-10 * sw[1] and itw <= itv
    assert np.abs(xv - xw).max() < 1e-8


def test_file_entry_points_check_arguments(tmp_path):
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.hb2_ell_read(ctypes.byref(h), str(tmp_path / "missing.ell").encode(), 0, None) == _lib.HB2_ERR_ARG
    assert b"not found" in lib.hb2_last_error()
    short = tmp_path / "short.ell"
    short.write_bytes(np.array([18, 2, 2, 32], "<u8").tobytes())
    assert lib.hb2_ell_read(ctypes.byref(h), str(short).encode(), 0, None) == _lib.HB2_ERR_ARG
    bad = tmp_path / "bad.ell"
    bad.write_bytes(np.array([10, 2, 2, 32, 1], "<u8").tobytes())     # size != stride * K
    assert lib.hb2_ell_read(ctypes.byref(h), str(bad).encode(), 0, None) == _lib.HB2_ERR_ARG
    trunc = tmp_path / "trunc.ell"
    trunc.write_bytes(np.array([32, 2, 2, 32, 1], "<u8").tobytes() + bytes(16))
    assert lib.hb2_ell_read(ctypes.byref(h), str(trunc).encode(), 0, None) == _lib.HB2_ERR_ARG
    assert lib.hb2_ell_read(None, b"x", 0, None) == _lib.HB2_ERR_ARG
    assert lib.hb2_ell_write(None, b"x") == _lib.HB2_ERR_ARG
    assert lib.hb2_ell_transpose(ctypes.byref(h), None, None) == _lib.HB2_ERR_ARG
