"""hb2_defect_ell_noalloc: the defect + squared-norm pass that allocates no device
memory, for callers that must not allocate (a hard device-memory budget with every
byte reserved up front, or a latency-critical loop where a cudaMalloc would stall
the device).  Its reduction scratch is a fixed device array inside the library.

Checked through the C ABI against hb2_defect_ell (which allocates its reduction
workspace on first use of a stream) on two calls in a row: the defect vector must
match bit for bit and the norm within the 1e-12 relative tolerance used for the
other reductions.  Kept in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

import honei_b200 as hb
from honei_b200 import _lib
from honei_b200.inputs import uniform

pytestmark = pytest.mark.gpu


def _defects(A, rhs, x, dtype, entry):
    n = A.rows()
    r = torch.zeros(n, dtype=dtype, device="cuda")
    nrm = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    _lib.call(entry, A.handle, ctypes.c_void_p(rhs.data_ptr()), ctypes.c_void_p(x.data_ptr()),
              ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(nrm.data_ptr()), None)
    torch.cuda.synchronize()
    return r.cpu().numpy(), nrm.item()


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


def test_noalloc_rejects_matrices_beyond_its_scratch():
    # level 12: 16,785,409 rows > 8,388,608 FP64 rows the static scratch covers
    A = hb.SparseMatrixELL.poisson_q1(12, torch.float64)
    n = A.rows()
    v = torch.zeros(n, dtype=torch.float64, device="cuda")
    nrm = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = _lib.load().hb2_defect_ell_noalloc(A.handle, ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                            ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(nrm.data_ptr()), None)
    assert st == _lib.HB2_ERR_UNSUPPORTED
    assert b"static scratch limit" in _lib.load().hb2_last_error()
