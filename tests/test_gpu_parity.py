"""Parity of the CUDA path (through the C ABI) with the oracle, which is itself pinned
bit-for-bit to the reference's tags::CPU outputs (test_oracle_golden.py).

Bit-exact: ELL/transfer assembly, SpMV, defect, Jacobi, banded Q1, matrix-free
transfers, element-wise BLAS-1, and the MG solve with the exact coarse CG.
Tolerances: tree-ordered reductions (dot, norm) within 1e-12 relative; CG
iteration counts within +-1 and the reference's stopping criterion met.
"""
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


# ----------------------------------------------------------------- assembly

@pytest.mark.parametrize("L", list(range(1, 10)))
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_q1_assembly_on_device_matches_reference_layout(oracle, L, dt):
    npdt = np.float64 if dt == torch.float64 else np.float32
    ref = oracle.q1_ell(L, npdt)
    A = SparseMatrixELL.poisson_q1(L, dt)
    assert (A.rows(), A.columns(), A.stride(), A.num_cols_per_row(), A.threads()) == (ref.rows, ref.cols, ref.stride, ref.K, 1)
    Aj, Ax, Arl = A.export()
    assert same_bits(Aj, ref.Aj) and same_bits(Ax, ref.Ax) and same_bits(Arl, ref.Arl)


@pytest.mark.parametrize("L", list(range(2, 10)))
def test_transfer_assembly_on_device(oracle, L):
    Pr, Rr = oracle.transfer_ell(L)
    P, R = SparseMatrixELL.transfer(L)
    for dev, ref in ((P, Pr), (R, Rr)):
        assert (dev.rows(), dev.columns(), dev.stride(), dev.num_cols_per_row()) == (ref.rows, ref.cols, ref.stride, ref.K)
        Aj, Ax, Arl = dev.export()
        assert same_bits(Aj, ref.Aj) and same_bits(Ax, ref.Ax) and same_bits(Arl, ref.Arl)


@pytest.mark.parametrize("L", [10, 11])
def test_assembly_at_levels_10_and_11(oracle, L):
    """The benchmark levels 10 and 11 (1,050,625 and 4,198,401 rows): operator and transfer
    matrices assembled on the device are the reference's arrays, bit for bit."""
    ref = oracle.q1_ell(L)
    A = SparseMatrixELL.poisson_q1(L)
    assert (A.rows(), A.columns(), A.stride(), A.num_cols_per_row()) == (ref.rows, ref.cols, ref.stride, ref.K)
    Aj, Ax, Arl = A.export()
    assert same_bits(Aj, ref.Aj) and same_bits(Ax, ref.Ax) and same_bits(Arl, ref.Arl)
    del A, Aj, Ax, Arl, ref
    Pr, Rr = oracle.transfer_ell(L)
    P, R = SparseMatrixELL.transfer(L)
    for dev, r in ((P, Pr), (R, Rr)):
        assert (dev.rows(), dev.columns(), dev.stride(), dev.num_cols_per_row()) == (r.rows, r.cols, r.stride, r.K)
        Aj, Ax, Arl = dev.export()
        assert same_bits(Aj, r.Aj) and same_bits(Ax, r.Ax) and same_bits(Arl, r.Arl)


@pytest.mark.parametrize("T", [1, 2, 3])
def test_upload_reference_arrays_roundtrip(oracle, T):
    ref = oracle.q1_ell(5, T=T)
    A = SparseMatrixELL.from_arrays(ref.rows, ref.cols, ref.stride, ref.K, ref.Aj, ref.Ax, ref.Arl, threads=T)
    Aj, Ax, Arl = A.export()
    assert same_bits(Aj, ref.Aj) and same_bits(Ax, ref.Ax) and same_bits(Arl, ref.Arl)
    x = oracle.uniform(ref.cols, 7)
    y = dvec(np.zeros(ref.rows))
    hb.Product.value(y, A, dvec(x))
    assert same_bits(host(y), oracle.ell_spmv(ref, x))


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_upload_and_export_with_an_odd_slot_count(oracle, dt):
    """stride * num_cols_per_row odd (stride = rows of a (2^L + 1)^2 grid): the
    uint64 row lengths after F32 values stay 8-byte aligned on the way in and out"""
    from honei_b200 import inputs
    rows, cols, stride, K, Aj, Ax, Arl = inputs.q1_coefficient_operator(inputs.element_coefficients(5, 3), dt)
    assert (K * stride) % 2 == 1
    A = SparseMatrixELL.from_arrays(rows, cols, stride, K, Aj, Ax, Arl)
    Aj2, Ax2, Arl2 = A.export()
    assert same_bits(Aj2, Aj) and same_bits(Ax2, Ax) and same_bits(Arl2, Arl)


def test_upload_rejects_bad_columns(oracle):
    ref = oracle.q1_ell(3)
    Aj = ref.Aj.copy()
    Aj[5] = ref.cols + 3
    with pytest.raises(hb.HoneiError):
        SparseMatrixELL.from_arrays(ref.rows, ref.cols, ref.stride, ref.K, Aj, ref.Ax, ref.Arl)


# ----------------------------------------------------------------- SpMV family

@pytest.mark.parametrize("L", [1, 2, 3, 5, 7, 9, 10])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_spmv_and_defect_bit_exact(oracle, L, dt):
    npdt = np.float64 if dt == torch.float64 else np.float32
    ref = oracle.q1_ell(L, npdt)
    A = SparseMatrixELL.poisson_q1(L, dt)
    x, rhs = oracle.uniform(ref.cols, 7, npdt), oracle.uniform(ref.rows, 11, npdt)
    y = dvec(np.zeros(ref.rows, npdt))
    hb.Product.value(y, A, dvec(x))
    assert same_bits(host(y), oracle.ell_spmv(ref, x))
    r = dvec(np.zeros(ref.rows, npdt))
    nrm = torch.zeros(1, dtype=torch.float64, device=DEV)
    hb.Defect.value(r, dvec(rhs), A, dvec(x), norm2_out=nrm)
    rr = oracle.ell_defect(ref, rhs, x)
    assert same_bits(host(r), rr)
    expect = float(np.dot(rr.astype(np.float64), rr.astype(np.float64)))
    assert abs(nrm.item() - expect) <= 1e-12 * max(expect, 1e-300)


def test_product_dot_and_add(oracle):
    from honei_b200 import _lib
    ref = oracle.q1_ell(8)
    A = SparseMatrixELL.poisson_q1(8)
    x = oracle.uniform(ref.cols, 3)
    y = dvec(np.zeros(ref.rows))
    dot = torch.zeros(1, dtype=torch.float64, device=DEV)
    xd = dvec(x)
    _lib.call("hb2_product_dot_ell", A.handle, xd.ptr, y.ptr, dot.data_ptr(), None)
    yr = oracle.ell_spmv(ref, x)
    assert same_bits(host(y), yr)
    assert abs(dot.item() - float(yr @ x)) <= 1e-12 * abs(float(yr @ x))
    z0 = oracle.uniform(ref.rows, 4)
    z = dvec(z0)
    _lib.call("hb2_product_add_ell", A.handle, xd.ptr, z.ptr, None)
    assert same_bits(host(z), z0 + yr)


def test_transfer_spmv_prolmat(oracle):
    for L in (3, 6, 9):
        Pr, Rr = oracle.transfer_ell(L)
        P, R = SparseMatrixELL.transfer(L)
        c, f = oracle.uniform(Pr.cols, 31), oracle.uniform(Rr.cols, 32)
        fine, coarse = dvec(np.zeros(Pr.rows)), dvec(np.zeros(Rr.rows))
        hb.Prolongation.value(fine, dvec(c), prolmat=P, method=hb.methods.PROLMAT)
        hb.Restriction.value(coarse, dvec(f), resmat=R, method=hb.methods.PROLMAT)
        assert same_bits(host(fine), oracle.ell_spmv(Pr, c))
        assert same_bits(host(coarse), oracle.ell_spmv(Rr, f))


def test_empty_matrix_and_vectors():
    from honei_b200 import _lib
    out = torch.full((1,), 7.0, dtype=torch.float64, device=DEV)
    e = torch.zeros(0, dtype=torch.float64, device=DEV)
    _lib.call("hb2_norm_l2", 0, e.data_ptr(), 0, 1, out.data_ptr(), None, None)
    torch.cuda.synchronize()
    assert out.item() == 0.0
    _lib.call("hb2_scaled_sum", 0, e.data_ptr(), e.data_ptr(), 2.0, 0, None)


# ----------------------------------------------------------------- banded Q1

@pytest.mark.parametrize("L", [1, 2, 4, 7, 10])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_q1_banded_bit_exact(oracle, L, dt):
    npdt = np.float64 if dt == torch.float64 else np.float32
    bands = oracle.q1_bands(L, npdt)
    Q = hb.BandedMatrixQx.from_bands(bands)
    Qd = hb.BandedMatrixQx.poisson_q1(L, dt)
    n = bands.shape[1]
    x, rhs = oracle.uniform(n, 7, npdt), oracle.uniform(n, 11, npdt)
    for M in (Q, Qd):
        y = dvec(np.zeros(n, npdt))
        hb.Product.value(y, M, dvec(x))
        assert same_bits(host(y), oracle.q1_spmv(bands, x))
        r = dvec(np.zeros(n, npdt))
        hb.Defect.value(r, dvec(rhs), M, dvec(x))
        assert same_bits(host(r), oracle.q1_defect(bands, rhs, x))


def test_q1_banded_unaligned_x(oracle):
    """x not 16-byte aligned -> plain-load path, same bits."""
    bands = oracle.q1_bands(6)
    n = bands.shape[1]
    Q = hb.BandedMatrixQx.from_bands(bands)
    x = oracle.uniform(n, 7)
    buf = torch.zeros(n + 1, dtype=torch.float64, device=DEV)
    buf[1:] = torch.from_numpy(x).to(DEV)
    xv = DenseVector(buf[1:])
    assert xv.elements.data_ptr() % 16 != 0
    y = dvec(np.zeros(n))
    hb.Product.value(y, Q, xv)
    assert same_bits(host(y), oracle.q1_spmv(bands, x))


# ----------------------------------------------------------------- BLAS-1

@pytest.mark.parametrize("n", [1, 31, 1000, 1 << 20])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_blas1_bit_exact(oracle, n, dt):
    a, b = oracle.uniform(n, 1, dt), oracle.uniform(n, 2, dt)
    s = dt(0.375)
    x = dvec(a)
    hb.ScaledSum.value(x, dvec(b), 0.375)
    assert same_bits(host(x), (a + s * b).astype(dt))
    r = dvec(np.zeros(n, dt))
    hb.ScaledSum.value(r, dvec(a), dvec(b), -1.25)
    assert same_bits(host(r), (dt(-1.25) * b + a).astype(dt))
    x = dvec(a)
    hb.Sum.value(x, dvec(b))
    assert same_bits(host(x), a + b)
    x = dvec(a)
    hb.Difference.value(x, dvec(b))
    assert same_bits(host(x), a - b)
    hb.Difference.value(r, dvec(a), dvec(b))
    assert same_bits(host(r), a - b)
    x = dvec(a)
    hb.Scale.value(x, 3.5)
    assert same_bits(host(x), a * dt(3.5))
    hb.ElementProduct.value(r, dvec(a), dvec(b))
    assert same_bits(host(r), a * b)
    hb.fill(r, 2.5)
    assert np.all(host(r) == dt(2.5))


@pytest.mark.parametrize("n", [1, 1000, 1 << 22])
def test_dot_norm_deterministic(oracle, n):
    a, b = oracle.uniform(n, 1), oracle.uniform(n, 2)
    da, db = dvec(a), dvec(b)
    d1 = hb.DotProduct.value(da, db)
    d2 = hb.DotProduct.value(da, db)
    assert d1 == d2
    exact = float(np.sum(a.astype(np.longdouble) * b.astype(np.longdouble)))
    assert abs(d1 - exact) <= 1e-12 * np.sum(np.abs(a * b))
    nrm = hb.Norm.value(da, root=True)
    assert abs(nrm - np.sqrt(float(np.sum(a.astype(np.longdouble) ** 2)))) <= 1e-12 * nrm
    assert hb.Norm.value(da, root=False) == hb.DotProduct.value(da, da)


def test_convert_roundtrip(oracle):
    a = oracle.uniform(12345, 9)
    f = dvec(np.zeros(12345, np.float32))
    hb.convert(f, dvec(a))
    assert same_bits(host(f), a.astype(np.float32))
    d = dvec(np.zeros(12345))
    hb.convert(d, f)
    assert same_bits(host(d), a.astype(np.float32).astype(np.float64))


# ----------------------------------------------------------------- matrix-free transfers

MASKS = [np.full(8, 2, np.uint64), np.zeros(8, np.uint64), np.array([2, 0, 2, 0, 0, 2, 2, 0], np.uint64)]


@pytest.mark.parametrize("L", [1, 2, 3, 6, 10])
@pytest.mark.parametrize("mi", range(3))
def test_matrix_free_transfers_bit_exact(oracle, L, mi):
    mask = MASKS[mi]
    nf, nc = oracle.q1_n(L), oracle.q1_n(L - 1) if L > 1 else 4
    if L == 1:
        nc = 4
    for dt in (np.float64, np.float32):
        c, f = oracle.uniform(nc, 31, dt), oracle.uniform(nf, 32, dt)
        fine, coarse = dvec(np.zeros(nf, dt)), dvec(np.zeros(nc, dt))
        hb.Prolongation.value(fine, dvec(c), mask)
        hb.Restriction.value(coarse, dvec(f), mask)
        assert same_bits(host(fine), oracle.prolongation(c, nf, mask))
        assert same_bits(host(coarse), oracle.restriction(f, nc, mask))


def test_matrix_free_equals_prolmat_plus_dirichlet(oracle):
    """ProlongationPROLMATTest (prolongation_TEST.cc:93-138): NONE == PROLMAT + Dirichlet."""
    L = 5
    Pr, _ = oracle.transfer_ell(L)
    c = oracle.uniform(Pr.cols, 3)
    fine = dvec(np.zeros(Pr.rows))
    hb.Prolongation.value(fine, dvec(c))
    via_mat = oracle.ell_spmv(Pr, c)
    m = oracle.q1_m(L)
    g = via_mat.reshape(m, m)
    g[0, :] = g[-1, :] = g[:, 0] = g[:, -1] = 0.0
    assert np.array_equal(host(fine), g.ravel())


# ----------------------------------------------------------------- smoother and solvers

@pytest.mark.parametrize("L", [3, 6, 9])
@pytest.mark.parametrize("sweeps", [1, 4])
def test_jacobi_bit_exact(oracle, L, sweeps):
    A = SparseMatrixELL.poisson_q1(L)
    P = hb.RISmoother.jacobi_precon(A, 0.7)
    b = oracle.uniform(A.rows(), 5)
    x0 = oracle.uniform(A.rows(), 6) * 0.1
    x = dvec(x0)
    hb.RISmoother.value(A, P, dvec(b), x, max_iters=sweeps)
    assert same_bits(host(x), oracle.jacobi_q1(L, b, x0, sweeps))


@pytest.mark.parametrize("L", [5, 7])
def test_cg_fp64_golden(oracle, golden, L):
    """Plain CG FP64, b = A u*, x0 = 0, tol 1e-8 (the CPU-sized CG workload, at L = 7)."""
    A = SparseMatrixELL.poisson_q1(L)
    b = golden.array(f"cg_L{L}.b") if L == 5 else oracle.ell_spmv(oracle.q1_ell(L), oracle.uniform(A.rows(), 42))
    x = dvec(np.zeros(A.rows()))
    _, used, defect = hb.CGSolver.value(A, None, dvec(b), x, 2000, 1e-8)
    ref_iters = golden.scalar(f"cg_L{L}.iters")
    assert abs(used - ref_iters) <= 1
    xs = host(x)
    relres = np.linalg.norm(b - oracle.ell_spmv(oracle.q1_ell(L), xs)) / np.linalg.norm(b)
    assert relres < 1.5e-8
    assert np.linalg.norm(xs - golden_x(golden, oracle, L)) / np.linalg.norm(xs) < 1e-6


def golden_x(golden, oracle, L):
    if f"cg_L{L}.x" in golden.full:
        return golden.array(f"cg_L{L}.x")
    return oracle.cg_q1(L, oracle.ell_spmv(oracle.q1_ell(L), oracle.uniform(oracle.q1_n(L), 42)))[0]


def test_cg_cooperative_path(oracle):
    """n > 4096 uses the cooperative whole-GPU kernel with bounded grid barriers."""
    L = 8
    ref = oracle.q1_ell(L)
    b = oracle.ell_spmv(ref, oracle.uniform(ref.rows, 42))
    A = SparseMatrixELL.poisson_q1(L)
    x = dvec(np.zeros(ref.rows))
    _, used, _ = hb.CGSolver.value(A, None, dvec(b), x, 3000, 1e-8)
    _, ref_used = oracle.cg_q1(L, b, max_iters=3000)
    assert abs(used - ref_used) <= 1
    xs = host(x)
    assert np.linalg.norm(b - oracle.ell_spmv(ref, xs)) / np.linalg.norm(b) < 1.5e-8


@pytest.mark.parametrize("L", [5, 6, 7])
def test_mg_bit_exact_with_reference(oracle, golden, L):
    """MG V(4,4) with the reference-order coarse CG reproduces the reference's
    tags::CPU iterates bit for bit (coarse cap 1000 as in the golden run)."""
    A = oracle.q1_ell(L)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42))
    data = hb.MGData.poisson_q1(3, L, params=hb.mg_params(max_iters_coarse=1000, eps=1e-10, coarse_exact=True))
    x = dvec(np.zeros(A.rows))
    hb.MGSolver.value(data, dvec(b), x)
    assert data.used_iters == golden.scalar(f"mg_L{L}.iters")
    assert data.used_iters_coarse == golden.scalar(f"mg_L{L}.coarse_iters")
    assert golden.matches(f"mg_L{L}.x", host(x))


def test_mg_level10(oracle):
    """Level 10, V(4,4), omega 0.7, coarse level 3 (cap 100), eps 1e-10."""
    L = 10
    A = oracle.q1_ell(L)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42))
    data = hb.MGData.poisson_q1(3, L, params=hb.mg_params(max_iters_coarse=100, eps=1e-10))
    x = dvec(np.zeros(A.rows))
    hb.MGSolver.value(data, dvec(b), x)
    xs = host(x)
    xo, it, _ = oracle.mg_q1(L, b, max_iters_coarse=100)
    assert data.used_iters == it
    assert same_bits(xs, xo)
    assert np.linalg.norm(b - oracle.ell_spmv(A, xs)) / np.linalg.norm(b) < 1e-10 * 1.0001 * data.rnorm_initial / np.linalg.norm(b) + 1e-9


def test_mg_f32(oracle, golden):
    A = oracle.q1_ell(6, np.float32)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42, np.float32))
    data = hb.MGData.poisson_q1(3, 6, dtype=torch.float32, params=hb.mg_params(max_iters_coarse=1000, eps=1e-5))
    x = dvec(np.zeros(A.rows, np.float32))
    hb.MGSolver.value(data, dvec(b), x)
    assert data.used_iters == golden.scalar("mg32_L6.iters")
    assert golden.matches("mg32_L6.x", host(x))


@pytest.mark.parametrize("L", [5, 6])
def test_ir_mixed(oracle, golden, L):
    """IRSolver FP64 outer / FP32 inner MG (inner eps 1e-3), reference semantics."""
    Ao = oracle.q1_ell(L)
    b = oracle.ell_spmv(Ao, oracle.uniform(Ao.rows, 42))
    A = SparseMatrixELL.poisson_q1(L)
    inner = hb.MGData.poisson_q1(3, L, dtype=torch.float32,
                                 params=hb.mg_params(max_iters_coarse=1000, eps=1e-3, coarse_exact=True))
    x = dvec(np.zeros(Ao.rows))
    _, it, st = hb.IRSolver.value(A, dvec(b), x, inner, eps=1e-10)
    assert abs(it - golden.scalar(f"ir_L{L}.iters")) <= 1
    xs = host(x)
    assert np.linalg.norm(b - oracle.ell_spmv(Ao, xs)) < 1e-10 * st[1] * 1.001
    xr, _, _ = oracle.ir_q1(L, b, max_iters_coarse=1000)
    assert np.linalg.norm(xs - xr) / np.linalg.norm(xr) < 1e-9


def test_mg_determinism():
    """Same inputs -> same bits, twice."""
    data = hb.MGData.poisson_q1(3, 8)
    n = ((1 << 8) + 1) ** 2
    b = torch.rand(n, dtype=torch.float64, device=DEV, generator=torch.Generator(device=DEV).manual_seed(3))
    out = []
    for _ in range(2):
        x = DenseVector(torch.zeros(n, dtype=torch.float64, device=DEV))
        hb.MGSolver.value(data, DenseVector(b), x)
        out.append(host(x))
    assert same_bits(out[0], out[1])


def test_mg_host_loop_mode_identical(monkeypatch):
    """HB2_MG_LOOP=host (loop on the host over the plain cycle graph) gives the same bits."""
    L = 7
    n = ((1 << L) + 1) ** 2
    data = hb.MGData.poisson_q1(3, L)
    b = DenseVector(torch.rand(n, dtype=torch.float64, device=DEV, generator=torch.Generator(device=DEV).manual_seed(5)))
    xs = []
    for mode in (None, "host"):
        if mode:
            monkeypatch.setenv("HB2_MG_LOOP", mode)
        x = DenseVector(torch.zeros(n, dtype=torch.float64, device=DEV))
        hb.MGSolver.value(data, b, x)
        xs.append((host(x), data.used_iters))
    assert xs[0][1] == xs[1][1]
    assert same_bits(xs[0][0], xs[1][0])


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_mg_fused_small_levels_identical(dt):
    """Small levels as cluster kernels give the same bits as one kernel per operator."""
    L = 9
    n = ((1 << L) + 1) ** 2
    b = DenseVector(torch.rand(n, dtype=dt, device=DEV, generator=torch.Generator(device=DEV).manual_seed(9)))
    out = []
    for fused in (True, False):
        data = hb.MGData.poisson_q1(3, L, dtype=dt, params=hb.mg_params(eps=1e-6 if dt == torch.float32 else 1e-10,
                                                                         fused_levels=fused))
        x = DenseVector(torch.zeros(n, dtype=dt, device=DEV))
        hb.MGSolver.value(data, b, x)
        out.append((host(x), data.used_iters))
    assert out[0][1] == out[1][1]
    assert same_bits(out[0][0], out[1][0])


def test_ir_mixed_fp64_coarse(oracle):
    """Mixed IR with an FP64 coarsest-level solve inside the FP32 inner MG:
    converges to the FP64 stop and agrees with the FP64 MG solution."""
    L = 7
    Ao = oracle.q1_ell(L)
    b = oracle.ell_spmv(Ao, oracle.uniform(Ao.rows, 42))
    A = SparseMatrixELL.poisson_q1(L)
    inner = hb.MGData.poisson_q1(3, L, dtype=torch.float32,
                                 params=hb.mg_params(eps=1e-3, coarse_eps=1e-10, coarse_exact=False, coarse_fp64=True))
    x = dvec(np.zeros(Ao.rows))
    _, it, st = hb.IRSolver.value(A, dvec(b), x, inner, eps=1e-10, reset_inner=True)
    xs = host(x)
    assert np.linalg.norm(b - oracle.ell_spmv(Ao, xs)) < 1e-10 * st[1] * 1.001
    x64, _, _ = oracle.mg_q1(L, b, max_iters_coarse=100)
    assert np.linalg.norm(xs - x64) / np.linalg.norm(x64) < 1e-6
    assert it <= 6


@pytest.mark.parametrize("layout", ["force2", "force4", "force8", "pattern1", "pattern2", "pattern4", "patternwin1",
                                    "patternwin2", "q1stencil2", "q1stencil4", "q1stencil8", "q1gather1",
                                    "q1gather2", "q1gather4", "q1pair", "q1strip2", "q1strip8"])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_compressed_layout_matches_plain(oracle, monkeypatch, dt, layout):
    """Value-dictionary + 16-bit offset layout (forceR) and row-pattern layout (patternR,
    square matrices, patternwinR with x staged in shared-memory windows, q1stencilR the
    Q1 stencil kernel; the rectangular transfers stay compressed): same bits as the plain
    layout (and the oracle) for every ELL kernel mode, square and rectangular."""
    from honei_b200 import _lib
    npdt = np.float64 if dt == torch.float64 else np.float32
    L = 9
    monkeypatch.setenv("HB2_ELL_COMPACT", layout)   # that layout, no autotuning
    monkeypatch.setenv("HB2_Q1_TRANSFER", "0")      # the transfers on their stored layout too
    A = SparseMatrixELL.poisson_q1(L, dt)
    P, R = SparseMatrixELL.transfer(L, dt)
    if layout.startswith("pattern") or layout.startswith("q1"):
        # two row patterns: interior stencil, Dirichlet identity row; 1 matrix byte per row
        assert A.layout() == (2, 2, 1)
        kern = {"patternwin": 1, "q1stencil": 2, "q1gather": 3, "q1pai": 4, "q1strip": 5}.get(layout[:-1], 0)
        want = (2, 2 if layout == "q1pair" else int(layout[-1]), kern)
    else:
        assert A.layout() == (1, 3, 27)
        want = (1, int(layout[-1]), 0)
    assert A.layout_variant(0) == want and A.layout_variant(1) == want
    assert P.layout()[0] == 1 and R.layout()[0] == 1
    monkeypatch.setenv("HB2_ELL_COMPACT", "0")
    A0 = SparseMatrixELL.poisson_q1(L, dt)
    P0, R0 = SparseMatrixELL.transfer(L, dt)
    assert A0.layout()[0] == 0 and P0.layout()[0] == 0
    n, nc = A.rows(), R.rows()
    x, b = oracle.uniform(n, 3, npdt), oracle.uniform(n, 4, npdt)
    c = oracle.uniform(nc, 5, npdt)
    Pj = hb.RISmoother.jacobi_precon(A0)
    outs = []
    for (M, Pm, Rm) in ((A, P, R), (A0, P0, R0)):
        y, r, s = dvec(np.zeros(n, npdt)), dvec(np.zeros(n, npdt)), dvec(np.zeros(n, npdt))
        hb.Product.value(y, M, dvec(x))
        nrm = torch.zeros(1, dtype=torch.float64, device=DEV)
        hb.Defect.value(r, dvec(b), M, dvec(x), norm2_out=nrm)
        bv, xv, cv = dvec(b), dvec(x), dvec(c)   # held until the launches have read them
        _lib.call("hb2_jacobi_sweep_ell", M.handle, Pj.ptr, bv.ptr, xv.ptr, s.ptr, None)
        f, cc = dvec(x.copy()), dvec(np.zeros(nc, npdt))
        _lib.call("hb2_product_add_ell", Pm.handle, cv.ptr, f.ptr, None)
        hb.Restriction.value(cc, dvec(x), resmat=Rm, method=hb.methods.PROLMAT)
        outs.append([host(v) for v in (y, r, s, f, cc)] + [nrm.item()])
    for a, b_ in zip(outs[0][:5], outs[1][:5]):
        assert same_bits(a, b_)
    # the fused norm's tree order follows the launch shape (rows per thread)
    assert abs(outs[0][5] - outs[1][5]) <= 1e-12 * outs[1][5]
    assert same_bits(outs[0][0], oracle.ell_spmv(oracle.q1_ell(L, npdt), x))


@pytest.mark.parametrize("L", [2, 3, 6, 10])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_q1_transfer_kernels_match_matrix_products(oracle, monkeypatch, L, dt):
    """The transfer matrices' products without reading them (y = P c, y += P c,
    y = R f) are the ELL kernels' and the oracle's bits."""
    from honei_b200 import _lib
    npdt = np.float64 if dt == torch.float64 else np.float32
    Pr, Rr = oracle.transfer_ell(L, npdt)
    P, R = SparseMatrixELL.transfer(L, dt)
    c, f, y0 = oracle.uniform(Pr.cols, 41, npdt), oracle.uniform(Pr.rows, 42, npdt), oracle.uniform(Pr.rows, 43, npdt)
    outs = []
    for flag in ("1", "0"):
        monkeypatch.setenv("HB2_Q1_TRANSFER", flag)
        yp, yr, ya = dvec(np.zeros(Pr.rows, npdt)), dvec(np.zeros(Rr.rows, npdt)), dvec(y0.copy())
        hb.Product.value(yp, P, dvec(c))
        hb.Product.value(yr, R, dvec(f))
        cv = dvec(c)
        _lib.call("hb2_product_add_ell", P.handle, cv.ptr, ya.ptr, None)
        outs.append([host(yp), host(yr), host(ya)])
    for a, b in zip(outs[0], outs[1]):
        assert same_bits(a, b)
    assert same_bits(outs[0][0], oracle.ell_spmv(Pr, c))
    assert same_bits(outs[0][1], oracle.ell_spmv(Rr, f))


def test_compressed_layout_falls_back_when_not_eligible(oracle):
    """More than 255 distinct values -> plain layout, still correct."""
    L = 8
    ref = oracle.q1_ell(L)
    Ax = ref.Ax.copy()
    nz = ref.Aj >= 0
    Ax[Ax != 0] = oracle.uniform(int((Ax != 0).sum()), 77) + 2.0   # many distinct values
    Arl = ref.Arl
    A = SparseMatrixELL.from_arrays(ref.rows, ref.cols, ref.stride, ref.K, ref.Aj, Ax, Arl)
    assert A.layout()[0] == 0
    ref2 = oracle.Ell(ref.rows, ref.cols, ref.stride, ref.K, 1, ref.Aj, Ax, Arl)
    x = oracle.uniform(ref.cols, 1)
    y = dvec(np.zeros(ref.rows))
    hb.Product.value(y, A, dvec(x))
    assert same_bits(host(y), oracle.ell_spmv(ref2, x))
