"""The C-ABI library loads without a GPU, exports every symbol include/honei_b200.h
declares, and rejects bad arguments before launching anything."""
import ctypes
import re
import subprocess

import numpy as np
import pytest
import torch

from honei_b200 import _lib
from honei_b200._lib import HB2_ERR_ARG, HB2_ERR_SIZE, HEADER, LIB_PATH


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"HB2_API[^;]*?\b(hb2_[a-z0-9_]+)\s*\(", text, flags=re.S)))


def test_library_loads():
    lib = _lib.load()
    assert lib.hb2_version().startswith(b"honei_b200")


def test_every_declared_symbol_is_exported():
    names = declared()
    assert len(names) >= 40
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (hb2_[a-z0-9_]+)$", out, flags=re.M))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = _lib.load()
    for n in names:
        assert getattr(lib, n) is not None
    # the Python binding knows every entry point
    assert set(names) <= set(_lib.SIGNATURES)


def test_argument_checks_without_gpu():
    lib = _lib.load()
    assert lib.hb2_ell_create(None, 0, 1, 1, 32, 1, 1, None, None, None, 1, None) == HB2_ERR_ARG
    assert b"bad argument" in lib.hb2_last_error()
    dummy = ctypes.c_void_p(16)
    # 10x10 is not a Q1 grid pair: size error before any launch
    assert lib.hb2_prolongation(0, dummy, 100, dummy, 25, None, None) == HB2_ERR_SIZE
    assert lib.hb2_restriction(0, dummy, 25, dummy, 100, None, None) == HB2_ERR_SIZE
    h = ctypes.c_void_p()
    assert lib.hb2_mg_create(ctypes.byref(h), 0, None, None, None, None, None) == HB2_ERR_ARG
    assert lib.hb2_q1_create(None, 0, 81, None, 1, None) == HB2_ERR_ARG
    assert lib.hb2_ell_layout(None, None, None, None) == HB2_ERR_ARG
    assert lib.hb2_ell_layout_variant(None, 0, None, None, None) == HB2_ERR_ARG
    # batched solver: coarse level above 3, or a system below the coarse level
    lv = (ctypes.c_uint32 * 2)(4, 2)
    assert lib.hb2_batch_create_q1(ctypes.byref(h), 1, lv, None, 4, None, None) == HB2_ERR_ARG
    assert lib.hb2_batch_create_q1(ctypes.byref(h), 2, lv, None, 3, None, None) == HB2_ERR_ARG
    assert b"level" in lib.hb2_last_error()


class _FakeMatrix:
    def __init__(self, rows, cols):
        self._r, self._c = rows, cols

    def rows(self):
        return self._r

    def columns(self):
        return self._c


def test_python_layer_size_checks_before_the_abi():
    """VectorSizeDoesNotMatch is raised before crossing the boundary (la/product.hh:155-162)."""
    from honei_b200 import Defect, DenseVector, Product, ScaledSum, VectorSizeDoesNotMatch
    x = DenseVector(torch.zeros(10, dtype=torch.float64), device="cpu")
    y = DenseVector(torch.zeros(9, dtype=torch.float64), device="cpu")
    with pytest.raises(VectorSizeDoesNotMatch):
        Product.value(y, _FakeMatrix(9, 9), x)
    with pytest.raises(VectorSizeDoesNotMatch):
        Defect.value(y, y, _FakeMatrix(9, 10), y)
    with pytest.raises(VectorSizeDoesNotMatch):
        ScaledSum.value(x, y, 2.0)


def test_error_mapping():
    from honei_b200._lib import HoneiError, VectorSizeDoesNotMatch, check
    lib = _lib.load()
    lib.hb2_prolongation(0, ctypes.c_void_p(16), 100, ctypes.c_void_p(16), 25, None, None)
    with pytest.raises(VectorSizeDoesNotMatch):
        check(HB2_ERR_SIZE)
    with pytest.raises(HoneiError):
        check(HB2_ERR_ARG)
