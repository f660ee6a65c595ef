"""The reference's FEAST MG test (math/mg_TEST.cc:398-463, MGSolverTestQuad) on the
device through the C ABI: its ELL files read by MatrixIO (hb2_ell_read), restriction
matrices by Transposition (hb2_ell_transpose), the W-cycle MG solve -- compared with
the reference's own solution and iteration counts, bit for bit; plus W-cycles on
the assembled Q1 hierarchy against the oracle."""
import numpy as np
import pytest
import torch

import honei_b200 as hb

pytestmark = pytest.mark.gpu


def read_all(feast, tmp_path, names, dtype=torch.float64):
    return [hb.MatrixIO.read_matrix(feast.write(tmp_path, n), dtype=dtype) for n in names]


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("name", ["A_1", "A_4", "A_6", "prol_2", "prol_6"])
def test_read_matrix(feast, oracle, tmp_path, name):
    A = read_all(feast, tmp_path, [name])[0]
    size, rows, cols, stride, K = feast.head(name)
    assert (A.rows(), A.columns(), A.stride(), A.num_cols_per_row(), A.threads()) == (rows, cols, stride, K, 1)
    Aj, Ax, Arl = A.export()
    assert np.array_equal(Aj, feast.z[name + ".Aj"].astype(np.uint64))
    assert same_bits(Ax, feast.z[name + ".Ax"])
    assert np.array_equal(Arl, feast.ell(oracle, name).Arl)


def test_read_matrix_float(feast, tmp_path):
    A = read_all(feast, tmp_path, ["A_5"], dtype=torch.float32)[0]
    _, Ax, _ = A.export()
    assert same_bits(Ax, feast.z["A_5.Ax"].astype(np.float32))


def test_write_matrix_round_trip(feast, tmp_path):
    A = read_all(feast, tmp_path, ["A_6"])[0]
    out = tmp_path / "out.ell"
    hb.MatrixIO.write_matrix(str(out), A)
    assert out.read_bytes() == feast.file_bytes("A_6")


@pytest.mark.parametrize("level", [2, 3, 4, 5, 6])
def test_transposition_is_the_reference_restriction(feast, tmp_path, level):
    P = read_all(feast, tmp_path, [f"prol_{level}"])[0]
    R = P.transposed()
    size, rows, cols, stride, K = feast.head(f"res_{level}")
    assert (R.rows(), R.columns(), R.stride(), R.num_cols_per_row()) == (rows, cols, stride, K)
    Aj, Ax, _ = R.export()
    assert np.array_equal(Aj, feast.z[f"res_{level}.Aj"].astype(np.uint64))
    assert same_bits(Ax, feast.z[f"res_{level}.Ax"])
    # the file the reference's own writer produced for this matrix
    out = tmp_path / "res.ell"
    hb.MatrixIO.write_matrix(str(out), R)
    assert out.read_bytes() == feast.file_bytes(f"res_{level}")


def feast_mg(feast, tmp_path, cycle):
    A = read_all(feast, tmp_path, [f"A_{i}" for i in range(1, 7)])
    P = read_all(feast, tmp_path, [f"prol_{i}" for i in range(2, 7)])
    R = [p.transposed() for p in P]
    prm = hb.mg_params(n_pre=4, n_post=4, max_iters=100, max_iters_coarse=100, eps=1e-8, omega=0.7, cycle=cycle)
    return hb.MGData(A, P, R, params=prm)


def test_feast_w_cycle_is_the_reference_solve(feast, tmp_path):
    mg = feast_mg(feast, tmp_path, "W")
    b = hb.VectorIO.read_vector(_exp(tmp_path, "rhs_6", feast))
    x = hb.VectorIO.read_vector(_exp(tmp_path, "init_6", feast))
    hb.MGSolver.value(mg, b, x)
    assert mg.used_iters == feast.meta["used_iters"]
    assert mg.used_iters_coarse == feast.meta["used_iters_coarse"]
    assert same_bits(x.numpy(), feast.z["ref_x"])
    assert np.abs(x.numpy() - feast.z["sol_6"]).max() < 8e-3     # the reference test's tolerance


def test_feast_v_cycle_matches_oracle(feast, oracle, tmp_path):
    mg = feast_mg(feast, tmp_path, "V")
    b = hb.DenseVector(feast.z["rhs_6"])
    x = hb.DenseVector(feast.z["init_6"])
    hb.MGSolver.value(mg, b, x)
    A = [feast.ell(oracle, f"A_{i}") for i in range(1, 7)]
    P = [feast.ell(oracle, f"prol_{i}") for i in range(2, 7)]
    R = [oracle.ell_transpose(p) for p in P]
    xo, it, stats = oracle.mg_ell(A, P, R, feast.z["rhs_6"], feast.z["init_6"], cycle="V", eps=1e-8)
    assert mg.used_iters == it and mg.used_iters_coarse == int(stats[3])
    assert same_bits(x.numpy(), xo)


def _exp(tmp_path, name, feast):
    """the vector as an EXP file (what VectorIO<io_formats::EXP> reads): %.17g per line"""
    path = tmp_path / name
    path.write_text("# " + name + "\n" + "".join("%.17g\n" % v for v in feast.z[name]))
    return str(path)


@pytest.mark.parametrize("dtype,L,lmin", [(torch.float64, 8, 2), (torch.float64, 10, 3), (torch.float32, 7, 2)])
def test_q1_w_cycle_matches_oracle(oracle, dtype, L, lmin):
    npdt = np.float64 if dtype == torch.float64 else np.float32
    n = oracle.q1_n(L)
    b = oracle.uniform(n, 5).astype(npdt)
    prm = hb.mg_params(eps=1e-6 if dtype == torch.float32 else 1e-10, max_iters_coarse=1000, cycle="W")
    mg = hb.MGData.poisson_q1(lmin, L, dtype=dtype, params=prm)
    x = hb.DenseVector(n, dtype=dtype)
    hb.MGSolver.value(mg, hb.DenseVector(b), x)
    xo, it, stats = oracle.mg_q1(L, b, min_level=lmin, max_iters_coarse=1000, eps=prm.eps_relative,
                                 coarse_eps=prm.coarse_eps, cycle="W")
    assert mg.used_iters == it and mg.used_iters_coarse == int(stats[3])
    assert same_bits(x.numpy(), xo)
