"""Launch shapes of the ELL kernels: blocks of 128, 256 or 512 threads (plain,
compressed and Q1 gather kernels; the plain kernel with one thread per row up to
256) and one or two threads per row (plain layout), pinned with HB2_ELL_BLOCK /
HB2_ELL_TPR or chosen by the autotuner.

Every shape forms the same products and slot-ordered sums, so every kernel mode is
the oracle's ELL product (la/product.hh:148-206) bit for bit; the fused norms
follow the launch shape's block order and stay within 1e-12 relative.  The
reference's own knobs are its block sizes (honei/honeirc:50-51) and the T threads
per row of its ELL kernel (backends/cuda/product.cu:148-200)."""
import ctypes

import numpy as np
import pytest
import torch

import honei_b200 as hb
from honei_b200 import DenseVector, SparseMatrixELL, _lib

pytestmark = pytest.mark.gpu

SHAPES = [(128, 1), (128, 2), (256, 2), (512, 2)]


def dvec(a):
    return DenseVector(torch.from_numpy(np.ascontiguousarray(a)).cuda())


def host(v):
    torch.cuda.synchronize()
    return v.numpy()


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def pin(monkeypatch, layout, bs, tpr):
    monkeypatch.setenv("HB2_ELL_COMPACT", layout)
    monkeypatch.setenv("HB2_ELL_BLOCK", str(bs))
    monkeypatch.setenv("HB2_ELL_TPR", str(tpr))


def check_square(oracle, A, ref, npdt, seed=3):
    """y = A x, r = b - A x with ||r||^2, y = A x with <y, x>, y += A x and the
    Jacobi sweep against the oracle"""
    n = ref.rows
    x, b = oracle.uniform(n, seed, npdt), oracle.uniform(n, seed + 1, npdt)
    xv, bv = dvec(x), dvec(b)
    y = dvec(np.zeros(n, npdt))
    hb.Product.value(y, A, xv)
    yr = oracle.ell_spmv(ref, x)
    assert same_bits(host(y), yr)
    r = dvec(np.zeros(n, npdt))
    nrm = torch.zeros(1, dtype=torch.float64, device="cuda")
    hb.Defect.value(r, bv, A, xv, norm2_out=nrm)
    rr = oracle.ell_defect(ref, b, x)
    assert same_bits(host(r), rr)
    e = float(np.dot(rr.astype(np.float64), rr.astype(np.float64)))
    assert abs(nrm.item() - e) <= 1e-12 * e
    dot = torch.zeros(1, dtype=torch.float64, device="cuda")
    y2 = dvec(np.zeros(n, npdt))
    _lib.call("hb2_product_dot_ell", A.handle, xv.ptr, y2.ptr, ctypes.c_void_p(dot.data_ptr()), None)
    assert same_bits(host(y2), yr)
    d = float(np.dot(yr.astype(np.float64), x.astype(np.float64)))
    assert abs(dot.item() - d) <= 1e-12 * np.dot(np.abs(yr.astype(np.float64)), np.abs(x.astype(np.float64)))
    z = dvec(b.copy())
    _lib.call("hb2_product_add_ell", A.handle, xv.ptr, z.ptr, None)
    assert same_bits(host(z), (b + yr).astype(npdt))
    P = hb.RISmoother.jacobi_precon(A, 0.7)
    s = dvec(np.zeros(n, npdt))
    _lib.call("hb2_jacobi_sweep_ell", A.handle, P.ptr, bv.ptr, xv.ptr, s.ptr, None)
    Ph = host(P)
    expect = (x + (Ph * (b - yr).astype(npdt)).astype(npdt)).astype(npdt)
    assert same_bits(host(s), expect)


@pytest.mark.parametrize("bs,tpr", SHAPES)
@pytest.mark.parametrize("L", [4, 7, 9])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_plain_shapes_bit_exact(oracle, monkeypatch, dt, L, bs, tpr):
    npdt = np.float64 if dt == torch.float64 else np.float32
    pin(monkeypatch, "0", bs, tpr)
    A = SparseMatrixELL.poisson_q1(L, dt)
    assert A.layout()[0] == 0 and A.launch_shape(0) == (bs, tpr) and A.launch_shape(1) == (bs, tpr)
    check_square(oracle, A, oracle.q1_ell(L, npdt), npdt)


@pytest.mark.parametrize("bs,tpr", SHAPES)
def test_plain_shapes_transfers(oracle, monkeypatch, bs, tpr):
    """The rectangular transfer matrices (K = 4 and 9) on their stored plain layout:
    y = P c, y += P c and y = R f with the cleared store"""
    pin(monkeypatch, "0", bs, tpr)
    monkeypatch.setenv("HB2_Q1_TRANSFER", "0")
    L = 8
    Pr, Rr = oracle.transfer_ell(L)
    P, R = SparseMatrixELL.transfer(L)
    assert P.launch_shape(0) == (bs, tpr)
    c, f, y0 = oracle.uniform(Pr.cols, 41), oracle.uniform(Pr.rows, 42), oracle.uniform(Pr.rows, 43)
    yp, ya, cc = dvec(np.zeros(Pr.rows)), dvec(y0.copy()), dvec(np.zeros(Rr.rows))
    cv, fv = dvec(c), dvec(f)
    hb.Product.value(yp, P, cv)
    _lib.call("hb2_product_add_ell", P.handle, cv.ptr, ya.ptr, None)
    hb.Restriction.value(cc, fv, resmat=R, method=hb.methods.PROLMAT)
    pc = oracle.ell_spmv(Pr, c)
    assert same_bits(host(yp), pc)
    assert same_bits(host(ya), y0 + pc)
    assert same_bits(host(cc), oracle.ell_spmv(Rr, f))


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_plain_one_thread_per_row_takes_at_most_256(oracle, monkeypatch, dt):
    """A pin of 512 threads with one thread per row runs the plain kernel in blocks
    of 256 (its launch bound), bit for bit"""
    npdt = np.float64 if dt == torch.float64 else np.float32
    pin(monkeypatch, "0", 512, 1)
    A = SparseMatrixELL.poisson_q1(7, dt)
    assert A.layout()[0] == 0 and A.launch_shape(0) == (256, 1) and A.launch_shape(1) == (256, 1)
    check_square(oracle, A, oracle.q1_ell(7, npdt), npdt)


def random_ell(oracle, rows, cols, seed, T=1):
    """rows of 0..12 entries at random columns: the runtime slot-count kernel"""
    rng = np.random.default_rng(seed)
    rp, ci, v = [0], [], []
    for r in range(rows):
        k = int(rng.integers(0, 13))
        cs = np.sort(rng.choice(cols, size=k, replace=False))
        ci += list(cs)
        v += list(rng.uniform(-1, 1, size=k))
        rp.append(len(ci))
    return oracle.ell_from_csr(rows, cols, np.array(rp, np.uint64), np.array(ci, np.uint64), np.array(v), T)


@pytest.mark.parametrize("bs,tpr", SHAPES + [(256, 1)])
@pytest.mark.parametrize("T", [1, 2])
def test_plain_shapes_runtime_slot_count(oracle, monkeypatch, bs, tpr, T):
    pin(monkeypatch, "0", bs, tpr)
    ref = random_ell(oracle, 6007, 5003, 11, T)
    A = SparseMatrixELL.from_arrays(ref.rows, ref.cols, ref.stride, ref.K, ref.Aj, ref.Ax, ref.Arl, threads=T)
    assert A.launch_shape(0) == (bs, tpr)
    x = oracle.uniform(ref.cols, 5)
    y = dvec(np.zeros(ref.rows))
    hb.Product.value(y, A, dvec(x))
    assert same_bits(host(y), oracle.ell_spmv(ref, x))


@pytest.mark.parametrize("layout", ["force2", "force8", "q1gather1", "q1gather4", "q1strip4"])
@pytest.mark.parametrize("bs", [128, 512])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_compressed_and_q1_gather_shapes(oracle, monkeypatch, dt, layout, bs):
    npdt = np.float64 if dt == torch.float64 else np.float32
    pin(monkeypatch, layout, bs, 2)     # threads per row stays 1 off the plain layout
    L = 9
    A = SparseMatrixELL.poisson_q1(L, dt)
    assert A.launch_shape(0) == (bs, 1) and A.launch_shape(1) == (bs, 1)
    assert A.layout_variant(0)[1] == int(layout[-1])
    check_square(oracle, A, oracle.q1_ell(L, npdt), npdt)


def test_fixed_shape_kernels_stay_at_256(monkeypatch):
    """The general row-pattern, windowed, bulk-copy and pair kernels keep 256 threads"""
    for layout in ("pattern2", "patternwin1", "q1stencil4", "q1pair"):
        pin(monkeypatch, layout, 512, 2)
        A = SparseMatrixELL.poisson_q1(9)
        assert A.launch_shape(0) == (256, 1), layout


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_mg_on_plain_shapes_bit_exact(oracle, monkeypatch, dt):
    """MG V(4,4) with the levels above the fused small-level kernels on the plain
    layout in blocks of 512, two threads per row: the oracle's iterates bit for bit
    (reference-order coarse CG), cycle count equal"""
    npdt = np.float64 if dt == torch.float64 else np.float32
    pin(monkeypatch, "0", 512, 2)
    L = 9
    A = oracle.q1_ell(L, npdt)
    b = oracle.ell_spmv(A, oracle.uniform(A.rows, 42, npdt))
    eps = 1e-10 if dt == torch.float64 else 1e-5
    data = hb.MGData.poisson_q1(3, L, dtype=dt, params=hb.mg_params(max_iters_coarse=100, eps=eps, coarse_exact=True))
    x = dvec(np.zeros(A.rows, npdt))
    hb.MGSolver.value(data, dvec(b), x)
    xo, it, _ = oracle.mg_q1(L, b, max_iters_coarse=100, eps=eps)
    assert data.used_iters == it
    assert same_bits(host(x), xo)


def test_batched_solve_on_plain_shapes(monkeypatch):
    """The batched PCG's work-list launches (levels 4..7 on the plain layout) in
    blocks of 128, two threads per row: every right-hand side converges"""
    pin(monkeypatch, "0", 128, 2)
    systems = [(4, 1), (6, 3), (7, 2), (5, 8)]
    B = hb.BatchedPoissonSolver(systems)
    for s, (level, k) in enumerate(systems):
        n = hb.BatchedPoissonSolver.unknowns(level)
        rhs = np.stack([np.random.default_rng(100 * s + j).uniform(-1, 1, n) for j in range(k)])
        B.set_rhs(s, torch.from_numpy(rhs).cuda())
    B.solve()
    torch.cuda.synchronize()
    for s, (level, k) in enumerate(systems):
        for j in range(k):
            it, rel = B.result(s, j)
            assert rel < 1e-8 and 0 < it < 100, (s, j, it, rel)


def test_tuner_times_the_shape_and_records_it(oracle, monkeypatch, tmp_path):
    """Without pins the autotuner picks a shape from the timed set (plain-only
    matrices from 4,096 rows up included) and appends it to HB2_TUNE_FILE."""
    for v in ("HB2_ELL_COMPACT", "HB2_ELL_BLOCK", "HB2_ELL_TPR"):
        monkeypatch.delenv(v, raising=False)
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("HB2_TUNE_FILE", str(path))
    ref = random_ell(oracle, 9001, 9001, 23)     # a shape no other test creates
    A = SparseMatrixELL.from_arrays(ref.rows, ref.cols, ref.stride, ref.K, ref.Aj, ref.Ax, ref.Arl)
    assert A.layout()[0] == 0
    for cls in (0, 1):
        bs, tpr = A.launch_shape(cls)
        assert bs in (128, 256, 512) and tpr in (1, 2)
    lines = [l.split() for l in path.read_text().splitlines()]
    mine = [l for l in lines if l[2] == "9001" and l[3] == "9001"]
    # device dtype rows cols K table patterns kind | layout rpt (x2) | block tpr (x2)
    assert len(mine) == 1 and len(mine[0]) == 16
    assert (int(mine[0][12]), int(mine[0][13])) == A.launch_shape(0)
    x = oracle.uniform(ref.cols, 9)
    y = dvec(np.zeros(ref.rows))
    hb.Product.value(y, A, dvec(x))
    assert same_bits(host(y), oracle.ell_spmv(ref, x))
    B = SparseMatrixELL.poisson_q1(10)
    kind, _, kernel = B.layout_variant(0)
    bs, tpr = B.launch_shape(0)
    assert tpr == 1 and bs in (128, 256, 512)
    if kind == 2 and kernel not in (3, 5):
        assert bs == 256      # row-pattern kernels other than the Q1 gather and strip forms
