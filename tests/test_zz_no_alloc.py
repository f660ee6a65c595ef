"""hb2_defect_ell_noalloc: the defect + squared-norm pass that allocates no device
memory.  It exists for callers that cannot call cudaMalloc: code running under a
hard device-memory budget where every byte is reserved up front, or a
latency-critical loop where an allocation would synchronise the device.  Its
reduction scratch is a fixed device array inside the library.

Checked through the C ABI:
  * the first call of the file runs on a stream nothing has used and creates no
    reduction workspace (the library's workspace count does not move);
  * against hb2_defect_ell (itself oracle-tested) on two calls in a row: the defect
    vector bit for bit, the norm within the 1e-12 relative tolerance used for the
    other reductions;
  * at level 11 (4,198,401 rows) against the oracle, also with the matrix pinned to
    the one-row-per-thread row-pattern layout, whose 16,400 row blocks exceed the
    scratch: the call must still succeed, so the answer depends on the row count
    alone;
  * beyond the row limit the call is refused before anything launches.
Kept in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

import honei_b200 as hb
from honei_b200 import _lib
from honei_b200.inputs import uniform

pytestmark = pytest.mark.gpu


def _defects(A, rhs, x, dtype, entry, stream=None):
    n = A.rows()
    r = torch.zeros(n, dtype=dtype, device="cuda")
    nrm = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    s = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    _lib.call(entry, A.handle, ctypes.c_void_p(rhs.data_ptr()), ctypes.c_void_p(x.data_ptr()),
              ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(nrm.data_ptr()), s)
    torch.cuda.synchronize()
    return r.cpu().numpy(), nrm.item()


def test_noalloc_first_call_creates_no_workspace():
    A = hb.SparseMatrixELL.poisson_q1(9, torch.float64)
    n = A.rows()
    rhs = torch.from_numpy(uniform(n, 3)).cuda()
    x = torch.from_numpy(uniform(n, 4)).cuda()
    fresh = torch.cuda.Stream()
    torch.cuda.synchronize()
    before = int(_lib.load().hb2_workspace_count())
    launches = hb.launch_count()
    r_new, n_new = _defects(A, rhs, x, torch.float64, "hb2_defect_ell_noalloc", fresh)
    assert int(_lib.load().hb2_workspace_count()) == before
    assert hb.launch_count() - launches >= 1    # the fused pass (and, on some layouts, its partials' sum)
    r_ref, n_ref = _defects(A, rhs, x, torch.float64, "hb2_defect_ell", fresh)
    assert int(_lib.load().hb2_workspace_count()) == before + 1   # the allocating entry point does create one
    assert np.array_equal(r_new.view(np.uint8), r_ref.view(np.uint8))
    assert abs(n_new - n_ref) <= 1e-12 * n_ref


@pytest.mark.parametrize("dtype,level", [(torch.float64, 9), (torch.float32, 10), (torch.float64, 3)])
def test_noalloc_defect_matches_allocating_entry_point(dtype, level):
    npdt = np.float64 if dtype == torch.float64 else np.float32
    A = hb.SparseMatrixELL.poisson_q1(level, dtype)
    n = A.rows()
    for call in range(2):   # two calls in a row: the shared scratch is reused
        rhs = torch.from_numpy(uniform(n, 11 + call, dtype=npdt)).cuda()
        x = torch.from_numpy(uniform(n, 7 + call, dtype=npdt)).cuda()
        r_ref, n_ref = _defects(A, rhs, x, dtype, "hb2_defect_ell")
        r_new, n_new = _defects(A, rhs, x, dtype, "hb2_defect_ell_noalloc")
        assert np.array_equal(r_new.view(np.uint8), r_ref.view(np.uint8))
        assert n_ref > 0
        assert abs(n_new - n_ref) <= 1e-12 * n_ref


@pytest.mark.parametrize("pin", [None, "pattern1"])
def test_noalloc_level11_against_the_oracle(pin, monkeypatch):
    from oracle import oracle as o
    if pin:
        monkeypatch.setenv("HB2_ELL_COMPACT", pin)
    A = hb.SparseMatrixELL.poisson_q1(11, torch.float64)
    n = A.rows()
    assert n == 4198401
    if pin:
        layout, rpt, _ = A.layout_variant(1)
        assert (layout, rpt) == (2, 1)   # row patterns, 16,400 row blocks at one row per thread
    rhs_h, x_h = uniform(n, 21), uniform(n, 22)
    rhs, x = torch.from_numpy(rhs_h).cuda(), torch.from_numpy(x_h).cuda()
    for call in range(2):
        r_new, n_new = _defects(A, rhs, x, torch.float64, "hb2_defect_ell_noalloc")
        r_ora = o.ell_defect(o.q1_ell(11), rhs_h, x_h) if call == 0 else r_ora
        assert np.array_equal(r_new.view(np.uint8), r_ora.view(np.uint8))
        n_ora = float(np.dot(r_ora, r_ora))
        assert abs(n_new - n_ora) <= 1e-12 * n_ora


def test_noalloc_rejects_matrices_beyond_its_scratch():
    # level 12: 16,785,409 rows > 8,388,608 FP64 rows the static scratch covers
    A = hb.SparseMatrixELL.poisson_q1(12, torch.float64)
    n = A.rows()
    v = torch.zeros(n, dtype=torch.float64, device="cuda")
    nrm = torch.zeros(1, dtype=torch.float64, device="cuda")
    launches = hb.launch_count()
    st = _lib.load().hb2_defect_ell_noalloc(A.handle, ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                            ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(nrm.data_ptr()), None)
    assert st == _lib.HB2_ERR_UNSUPPORTED
    assert b"static scratch limit" in _lib.load().hb2_last_error()
    assert hb.launch_count() == launches
