"""The legacy banded Multigrid on the device through the C ABI: the reference's own
solutions on its FEAST banded test data, bit for bit, and larger assembled Q1
hierarchies against the oracle, bit for bit with the same cycle counts."""
import numpy as np
import pytest
import torch

import honei_b200 as hb

from test_legacy_mg_host import CASES, levels

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def device_levels(bands):
    return [hb.BandedMatrixQx.from_bands(bands[l].reshape(9, -1)) for l in sorted(bands)]


def info_of(kw):
    return hb.mg_info(n_max_iter=kw.get("n_max_iter", 16), initial_zero=kw.get("initial_zero", True),
                      convergence_check=kw.get("convergence_check", False), is_smoother=kw.get("is_smoother", False),
                      tolerance=kw.get("tolerance", 1e-8), n_pre_smooth=kw.get("n_pre", 2),
                      adapt_correction_factor=kw.get("adapt", 1.0), macro_border_mask=kw.get("mask"))


@pytest.fixture(scope="module")
def lmg_golden():
    import os
    return dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_legacy_mg.npz")))


@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_cases(lmg_golden, oracle, case):
    c = CASES[case]
    bands, b = levels(lmg_golden, c["L"], c["dtype"])
    n = b.size
    x0 = (oracle.uniform(n, c["x0"]) if c["x0"] else np.zeros(n)).astype(c["dtype"])
    mg = hb.Multigrid(device_levels(bands), 1, info_of(c["kw"]))
    x, cycles, _ = mg.value(hb.DenseVector(b), hb.DenseVector(x0))
    assert same_bits(x.numpy(), lmg_golden[f"lmg_{case}.x"])
    assert cycles == oracle.legacy_mg(bands, b, x0, **c["kw"])[1]


@pytest.mark.parametrize("dtype,L,lmin", [(np.float64, 8, 1), (np.float64, 9, 2), (np.float32, 8, 1)])
@pytest.mark.parametrize("initial_zero", [True, False])
def test_assembled_hierarchy(oracle, dtype, L, lmin, initial_zero):
    bands = {l: oracle.q1_bands(l, dtype).reshape(-1) for l in range(lmin, L + 1)}
    n = oracle.q1_n(L)
    b = oracle.q1_spmv(bands[L].reshape(9, -1), oracle.uniform(n, 3).astype(dtype))
    x0 = (0.01 * oracle.uniform(n, 4)).astype(dtype)
    kw = dict(n_max_iter=40, initial_zero=initial_zero, tolerance=1e-6 if dtype == np.float32 else 1e-10, n_pre=2)
    xo, co = oracle.legacy_mg(bands, b, x0, **kw)
    td = torch.float64 if dtype == np.float64 else torch.float32
    mg = hb.Multigrid([hb.BandedMatrixQx.poisson_q1(l, td) for l in range(lmin, L + 1)], lmin, info_of(kw))
    x, cycles, _ = mg.value(hb.DenseVector(b), hb.DenseVector(x0))
    assert cycles == co
    assert same_bits(x.numpy(), xo)


def test_handle_reuse(lmg_golden):
    c = CASES["A"]
    bands, b = levels(lmg_golden, 5, np.float64)
    mg = hb.Multigrid(device_levels(bands), 1, info_of(c["kw"]))
    x1 = mg.value(hb.DenseVector(b), hb.DenseVector(b.size))[0].numpy()
    x2 = mg.value(hb.DenseVector(b), hb.DenseVector(b.size))[0].numpy()
    assert same_bits(x1, x2) and same_bits(x1, lmg_golden["lmg_A.x"])


@pytest.mark.parametrize("case", ["E", "F"])
def test_mixed(lmg_golden, oracle, case):
    """Multigrid<..., MIXED>: the inner FP32 cycles are bit-identical; the outer FP64 norm
    (a tree reduction here, sequential in the reference) also scales the defect, so the
    result agrees to rounding and the step counts agree exactly."""
    from test_legacy_mg_host import MIXED_CASES, mixed_levels
    c = MIXED_CASES[case]
    b32, a64, b = mixed_levels(lmg_golden)
    x0 = oracle.uniform(b.size, c["x0"]) if c["x0"] else np.zeros(b.size)
    xo, outer_o, inner_o = oracle.legacy_mg_mixed(b32, a64, b, x0, adapt=c["adapt"])
    info = hb.mg_info(n_max_iter=2, adapt_correction_factor=c["adapt"], adaptive=True)
    mg = hb.Multigrid(device_levels(b32), 1, info)
    A64 = hb.BandedMatrixQx.from_bands(a64.reshape(9, -1))
    x, outer, inner, _ = mg.value_mixed(A64, hb.DenseVector(b), hb.DenseVector(x0))
    assert (outer, inner) == (outer_o, inner_o)
    ref = lmg_golden[f"lmg_{case}.x"]
    assert np.abs(x.numpy() - ref).max() <= 1e-9 * np.abs(ref).max()
    assert np.abs(x.numpy() - lmg_golden["bin_1089"][11]).max() < 1e-4


def test_mixed_assembled_level9(oracle):
    """FP32 levels 1-9 under FP64 defect correction on the assembled Q1 operator"""
    L = 9
    b32 = {l: oracle.q1_bands(l, np.float32).reshape(-1) for l in range(1, L + 1)}
    a64 = oracle.q1_bands(L, np.float64)
    b = oracle.q1_spmv(a64, oracle.uniform(oracle.q1_n(L), 3))
    xo, outer_o, inner_o = oracle.legacy_mg_mixed(b32, a64.reshape(-1), b, np.zeros(b.size), n_max_iter=4)
    mg = hb.Multigrid([hb.BandedMatrixQx.poisson_q1(l, torch.float32) for l in range(1, L + 1)], 1,
                      hb.mg_info(n_max_iter=4, adaptive=True))
    x, outer, inner, _ = mg.value_mixed(hb.BandedMatrixQx.poisson_q1(L), hb.DenseVector(b), hb.DenseVector(b.size))
    assert (outer, inner) == (outer_o, inner_o)
    assert np.abs(x.numpy() - xo).max() <= 1e-9 * np.abs(xo).max()
