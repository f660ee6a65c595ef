"""HONEI's linear-algebra layer for the B200 tag: containers and operators.

Mirrors the reference's tag-dispatched API (``Product<Tag>::value(y, A, x)``
etc.) with the same argument order, meaning and size checks; every operator is
one call into libhonei_b200.so.  Device buffers are torch CUDA tensors; torch is
used only to own memory and to name the current stream.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import HB2_F32, HB2_F64, VectorSizeDoesNotMatch, call

_DT = {torch.float64: HB2_F64, torch.float32: HB2_F32}
_NP = {HB2_F64: np.float64, HB2_F32: np.float32}
_TORCH = {HB2_F64: torch.float64, HB2_F32: torch.float32}


class tags:
    """Tag of the new backend (util/tags.hh pattern): ``name = "b200"``."""

    class B200:
        name = "b200"


def _stream(stream=None) -> ctypes.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def dtype_code(dtype) -> int:
    if isinstance(dtype, torch.dtype):
        return _DT[dtype]
    return {np.dtype(np.float64): HB2_F64, np.dtype(np.float32): HB2_F32}[np.dtype(dtype)]


class DenseVector:
    """DenseVector<DT> resident on the device (la/dense_vector.hh)."""

    def __init__(self, data, dtype=None, device="cuda"):
        if isinstance(data, DenseVector):
            data = data.elements
        if isinstance(data, (int, np.integer)):
            self.elements = torch.zeros(int(data), dtype=dtype or torch.float64, device=device)
        elif isinstance(data, torch.Tensor):
            self.elements = data if data.is_cuda else data.to(device)
            if dtype is not None:
                self.elements = self.elements.to(dtype)
            self.elements = self.elements.contiguous()
        else:
            arr = np.ascontiguousarray(data)
            t = torch.from_numpy(arr)
            if dtype is not None:
                t = t.to(dtype)
            self.elements = t.to(device)

    def size(self) -> int:
        return self.elements.numel()

    def __len__(self) -> int:
        return self.size()

    @property
    def dtype(self) -> int:
        return _DT[self.elements.dtype]

    @property
    def ptr(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(self.elements.data_ptr())

    def copy(self) -> "DenseVector":
        return DenseVector(self.elements.clone())

    def numpy(self) -> np.ndarray:
        return self.elements.detach().cpu().numpy()


def _vec(v) -> DenseVector:
    return v if isinstance(v, DenseVector) else DenseVector(v)


class SparseMatrixELL:
    """SparseMatrixELL<DT> on the device (la/sparse_matrix_ell.hh:44-129).

    Built from the reference's arrays (Aj, Ax, Arl, stride, num_cols_per_row,
    threads) or assembled on the device (``poisson_q1``, ``transfer``)."""

    def __init__(self, handle: int, owner=True):
        self._h = ctypes.c_void_p(handle)
        self._owner = owner
        rows, cols, stride, K, T, nbytes = (ctypes.c_uint64() for _ in range(6))
        call("hb2_ell_info", self._h, ctypes.byref(rows), ctypes.byref(cols), ctypes.byref(stride),
             ctypes.byref(K), ctypes.byref(T), ctypes.byref(nbytes))
        self._rows, self._cols = rows.value, cols.value
        self._stride, self._K, self._T, self.device_bytes = stride.value, K.value, T.value, nbytes.value
        self._dtype = None

    @classmethod
    def from_arrays(cls, rows, columns, stride, num_cols_per_row, Aj, Ax, Arl, threads=1, stream=None):
        Aj = np.ascontiguousarray(Aj, np.uint64)
        Ax = np.ascontiguousarray(Ax)
        Arl = np.ascontiguousarray(Arl, np.uint64)
        if Aj.size != num_cols_per_row * stride or Ax.size != num_cols_per_row * stride or Arl.size != rows:
            raise VectorSizeDoesNotMatch(_lib.HB2_ERR_SIZE, "ELL arrays do not match stride * num_cols_per_row")
        h = ctypes.c_void_p()
        call("hb2_ell_create", ctypes.byref(h), dtype_code(Ax.dtype), rows, columns, stride, num_cols_per_row,
             threads, Aj.ctypes.data_as(ctypes.c_void_p), Ax.ctypes.data_as(ctypes.c_void_p),
             Arl.ctypes.data_as(ctypes.c_void_p), 1, _stream(stream))
        m = cls(h.value)
        m._dtype = dtype_code(Ax.dtype)
        return m

    @classmethod
    def poisson_q1(cls, level: int, dtype=torch.float64, aniso: float = 1.0, stream=None):
        """FillMatrix<POISSON, DIRICHLET_0> at grid level L as ELL (assembled on the device)."""
        h = ctypes.c_void_p()
        call("hb2_ell_create_q1", ctypes.byref(h), dtype_code(dtype), level, aniso, _stream(stream))
        m = cls(h.value)
        m._dtype = dtype_code(dtype)
        return m

    @classmethod
    def transfer(cls, fine_level: int, dtype=torch.float64, stream=None):
        """(P, R): ProlongationMatrix (level-1 -> level) and its Transposition."""
        p, r = ctypes.c_void_p(), ctypes.c_void_p()
        call("hb2_ell_create_transfer", ctypes.byref(p), ctypes.byref(r), dtype_code(dtype), fine_level,
             _stream(stream))
        P, R = cls(p.value), cls(r.value)
        P._dtype = R._dtype = dtype_code(dtype)
        return P, R

    @classmethod
    def _from_handle(cls, h, dtype):
        m = cls(h.value)
        m._dtype = dtype_code(dtype)
        return m

    def transposed(self, stream=None) -> "SparseMatrixELL":
        """Transposition<tags::B200>::value(A) (math/transposition.hh:36-50)."""
        h = ctypes.c_void_p()
        call("hb2_ell_transpose", ctypes.byref(h), self._h, _stream(stream))
        m = SparseMatrixELL(h.value)
        m._dtype = self._dtype
        return m

    def to_bf16(self, compensate: bool = False, stream=None) -> "SparseMatrixELL":
        """A BF16-stored copy (hb2_ell_create_bf16): entries bf16(s * a) with one
        scale s per matrix, FP32 accumulation and one division by s per row; with
        compensate=True the diagonal in FP32, absorbing the row's off-diagonal
        rounding errors (row sums kept).  An F32 matrix; ``scale`` and
        ``max_rel_error`` describe the rounding."""
        h = ctypes.c_void_p()
        s, e = ctypes.c_double(), ctypes.c_double()
        call("hb2_ell_create_bf16", ctypes.byref(h), self._h, 1 if compensate else 0, ctypes.byref(s),
             ctypes.byref(e), _stream(stream))
        m = SparseMatrixELL(h.value)
        m._dtype = dtype_code(torch.float32)
        m.scale, m.max_rel_error, m.compensated = s.value, e.value, bool(compensate)
        return m

    def converted(self, dtype, stream=None) -> "SparseMatrixELL":
        h = ctypes.c_void_p()
        call("hb2_ell_convert", ctypes.byref(h), self._h, dtype_code(dtype), _stream(stream))
        m = SparseMatrixELL(h.value)
        m._dtype = dtype_code(dtype)
        return m

    def rows(self) -> int:
        return self._rows

    def columns(self) -> int:
        return self._cols

    def layout(self):
        """(kind, table_size, matrix_bytes_per_row) of the device layout the
        matrix-vector kernels run on; kind 0 plain, 1 compressed (value codes +
        16-bit offsets), 2 row patterns."""
        c, t, rb = ctypes.c_int(), ctypes.c_uint32(), ctypes.c_uint32()
        call("hb2_ell_layout", self._h, ctypes.byref(c), ctypes.byref(t), ctypes.byref(rb))
        return c.value, t.value, rb.value

    def layout_variant(self, cls: int = 0):
        """(kind, rows_per_thread, kernel) of the kernel behind layout() for kernel
        class cls (0: products, sweeps, transfers; 1: defects with a fused norm);
        kernel 1 for the row-pattern kernel that stages x in shared-memory windows,
        2 for the Q1 stencil kernel (row patterns holding the full nine-point
        stencil, x windows staged by bulk copies), 3 for its gather form (plain
        loads), 4 for its pair form (two adjacent rows per thread), 5 for its strip
        form (rows_per_thread grid rows of one column per thread), 0 otherwise."""
        k, r, w = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        call("hb2_ell_layout_variant", self._h, cls, ctypes.byref(k), ctypes.byref(r), ctypes.byref(w))
        return k.value, r.value, w.value

    def launch_shape(self, cls: int = 0):
        """(threads_per_block, threads_per_row) of that kernel: the autotuner's
        choice among 128 / 256 / 512 threads (plain, compressed and Q1 gather
        kernels, the plain one with one thread per row up to 256; 256 for the
        others) and 1 or 2 threads per row (plain layout)."""
        b, t = ctypes.c_int(), ctypes.c_int()
        call("hb2_ell_launch_shape", self._h, cls, ctypes.byref(b), ctypes.byref(t))
        return b.value, t.value

    def stride(self) -> int:
        return self._stride

    def num_cols_per_row(self) -> int:
        return self._K

    def threads(self) -> int:
        return self._T

    @property
    def dtype(self) -> int:
        return self._dtype

    def export(self):
        """(Aj, Ax, Arl) in the reference layout, as host arrays."""
        torch.cuda.synchronize()
        n = self._K * self._stride
        Aj = np.zeros(n, np.uint64)
        Ax = np.zeros(n, _NP[self._dtype])
        Arl = np.zeros(self._rows, np.uint64)
        call("hb2_ell_export", self._h, Aj.ctypes.data_as(ctypes.c_void_p), Ax.ctypes.data_as(ctypes.c_void_p),
             Arl.ctypes.data_as(ctypes.c_void_p))
        return Aj, Ax, Arl

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def __del__(self):
        try:
            if self._owner and self._h:
                _lib.load().hb2_ell_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass


class BandedMatrixQx:
    """BandedMatrixQx<Q1Type, DT> on the device (la/banded_matrix_qx.hh:42-117)."""

    def __init__(self, handle, n, dtype):
        self._h = ctypes.c_void_p(handle)
        self._n = n
        self._dtype = dtype

    @classmethod
    def from_bands(cls, bands: np.ndarray, stream=None):
        bands = np.ascontiguousarray(bands)
        n = bands.shape[1]
        h = ctypes.c_void_p()
        call("hb2_q1_create", ctypes.byref(h), dtype_code(bands.dtype), n, bands.ctypes.data_as(ctypes.c_void_p), 1,
             _stream(stream))
        return cls(h.value, n, dtype_code(bands.dtype))

    @classmethod
    def poisson_q1(cls, level: int, dtype=torch.float64, aniso: float = 1.0, stream=None):
        h = ctypes.c_void_p()
        call("hb2_q1_create_poisson", ctypes.byref(h), dtype_code(dtype), level, aniso, _stream(stream))
        m = (1 << level) + 1
        return cls(h.value, m * m, dtype_code(dtype))

    def rows(self) -> int:
        return self._n

    def columns(self) -> int:
        return self._n

    @property
    def handle(self):
        return self._h

    def __del__(self):
        try:
            if self._h:
                _lib.load().hb2_q1_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass


def _check_size(a: int, b: int):
    if a != b:
        raise VectorSizeDoesNotMatch(_lib.HB2_ERR_SIZE, f"VectorSizeDoesNotMatch: {a} != {b}")


class SparseMatrixCSR:
    """SparseMatrixCSR<DT> on the device (la/sparse_matrix_csr.hh:44-125): Ar block
    offsets, Aj first column of each block, Ax csr::blocksize values per block."""

    def __init__(self, handle: int, dtype=None):
        self._h = ctypes.c_void_p(handle)
        rows, cols, bs, nb, nbytes = (ctypes.c_uint64() for _ in range(5))
        call("hb2_csr_info", self._h, ctypes.byref(rows), ctypes.byref(cols), ctypes.byref(bs), ctypes.byref(nb),
             ctypes.byref(nbytes))
        self._rows, self._cols, self._bs, self._nblocks = rows.value, cols.value, bs.value, nb.value
        self.device_bytes = nbytes.value
        self._dtype = dtype

    @classmethod
    def from_arrays(cls, rows, columns, Ar, Aj, Ax, blocksize=1, stream=None):
        """SparseMatrixCSR(blocksize, rows, columns, Aj, Ax, Ar, used) with host arrays."""
        Ar = np.ascontiguousarray(Ar, np.uint64)
        Ax = np.ascontiguousarray(Ax)
        if Ar.size != rows + 1:
            raise VectorSizeDoesNotMatch(_lib.HB2_ERR_SIZE, "Ar must hold rows + 1 offsets")
        nb = int(Ar[-1])
        Aj = np.ascontiguousarray(np.asarray(Aj)[:nb], np.uint64)
        if Aj.size != nb or Ax.size < nb * blocksize:
            raise VectorSizeDoesNotMatch(_lib.HB2_ERR_SIZE, "Aj / Ax shorter than Ar[rows] blocks")
        h = ctypes.c_void_p()
        call("hb2_csr_create", ctypes.byref(h), dtype_code(Ax.dtype), rows, columns, blocksize,
             Ar.ctypes.data_as(ctypes.c_void_p), Aj.ctypes.data_as(ctypes.c_void_p),
             Ax.ctypes.data_as(ctypes.c_void_p), 1, _stream(stream))
        return cls(h.value, dtype_code(Ax.dtype))

    @classmethod
    def from_ell(cls, A: "SparseMatrixELL", blocksize=1, stream=None):
        """SparseMatrixCSR(SparseMatrixELL) with csr::blocksize = blocksize."""
        h = ctypes.c_void_p()
        call("hb2_csr_from_ell", ctypes.byref(h), A.handle, blocksize, _stream(stream))
        return cls(h.value, A.dtype)

    def rows(self) -> int:
        return self._rows

    def columns(self) -> int:
        return self._cols

    def blocksize(self) -> int:
        return self._bs

    def used_blocks(self) -> int:
        return self._nblocks

    @property
    def dtype(self) -> int:
        return self._dtype

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def layout(self):
        """(slots, long_rows, long_entries, unroll) of the device layout: slot-major
        32-row slices of the rows of at most 128 entries (slots incl. padding) and
        128-entry chunks of the longer rows."""
        sl, lr, le, u = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        call("hb2_csr_layout", self._h, ctypes.byref(sl), ctypes.byref(lr), ctypes.byref(le), ctypes.byref(u))
        return sl.value, lr.value, le.value, u.value

    def export(self):
        """(Ar, Aj, Ax) as host arrays."""
        torch.cuda.synchronize()
        Ar = np.zeros(self._rows + 1, np.uint64)
        Aj = np.zeros(self._nblocks, np.uint64)
        Ax = np.zeros(self._nblocks * self._bs, _NP[self._dtype])
        call("hb2_csr_export", self._h, Ar.ctypes.data_as(ctypes.c_void_p), Aj.ctypes.data_as(ctypes.c_void_p),
             Ax.ctypes.data_as(ctypes.c_void_p))
        return Ar, Aj, Ax

    def __del__(self):
        try:
            if self._h:
                _lib.load().hb2_csr_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass


class Product:
    """Product<tags::B200>::value (la/product.hh)."""

    @staticmethod
    def value(y, A, x, stream=None):
        y, x = _vec(y), _vec(x)
        if isinstance(A, DenseVector):      # element-wise product r = a (.) b (la/product.hh:1198-1204)
            return ElementProduct.value(y, A, x, stream)
        _check_size(x.size(), A.columns())
        _check_size(A.rows(), y.size())
        if isinstance(A, BandedMatrixQx):
            call("hb2_product_q1", A.handle, x.ptr, y.ptr, _stream(stream))
        elif isinstance(A, SparseMatrixCSR):
            call("hb2_product_csr", A.handle, x.ptr, y.ptr, _stream(stream))
        else:
            call("hb2_product_ell", A.handle, x.ptr, y.ptr, _stream(stream))
        return y


class Defect:
    """Defect<tags::B200>::value(r, rhs, A, x) = rhs - A x (math/defect.hh)."""

    @staticmethod
    def value(r, rhs, A, x, norm2_out: torch.Tensor | None = None, stream=None):
        r, rhs, x = _vec(r), _vec(rhs), _vec(x)
        _check_size(x.size(), A.columns())
        if isinstance(A, SparseMatrixCSR):
            _check_size(rhs.size(), A.rows())
            _check_size(r.size(), A.rows())
            call("hb2_defect_csr", A.handle, rhs.ptr, x.ptr, r.ptr, _stream(stream))
            return r
        _check_size(rhs.size(), A.columns())
        _check_size(r.size(), A.rows())
        if isinstance(A, BandedMatrixQx):
            call("hb2_defect_q1", A.handle, rhs.ptr, x.ptr, r.ptr, _stream(stream))
        else:
            nptr = ctypes.c_void_p(norm2_out.data_ptr()) if norm2_out is not None else None
            call("hb2_defect_ell", A.handle, rhs.ptr, x.ptr, r.ptr, nptr, _stream(stream))
        return r


class ScaledSum:
    """ScaledSum<tags::B200>: value(x, y, b): x += b*y; value(r, x, y, b): r = b*y + x."""

    @staticmethod
    def value(*args, stream=None):
        if len(args) == 3:
            x, y, b = _vec(args[0]), _vec(args[1]), args[2]
            _check_size(x.size(), y.size())
            call("hb2_scaled_sum", x.dtype, x.ptr, y.ptr, float(b), x.size(), _stream(stream))
            return x
        r, x, y, b = _vec(args[0]), _vec(args[1]), _vec(args[2]), args[3]
        _check_size(x.size(), y.size())
        _check_size(x.size(), r.size())
        call("hb2_scaled_sum3", r.dtype, r.ptr, x.ptr, y.ptr, float(b), r.size(), _stream(stream))
        return r


class Sum:
    @staticmethod
    def value(x, y, stream=None):
        x, y = _vec(x), _vec(y)
        _check_size(x.size(), y.size())
        call("hb2_sum", x.dtype, x.ptr, y.ptr, x.size(), _stream(stream))
        return x


class Difference:
    @staticmethod
    def value(*args, stream=None):
        if len(args) == 2:
            x, y = _vec(args[0]), _vec(args[1])
            _check_size(x.size(), y.size())
            call("hb2_difference", x.dtype, x.ptr, y.ptr, x.size(), _stream(stream))
            return x
        r, x, y = (_vec(a) for a in args)
        _check_size(x.size(), y.size())
        _check_size(r.size(), x.size())
        call("hb2_difference3", r.dtype, r.ptr, x.ptr, y.ptr, r.size(), _stream(stream))
        return r


class Scale:
    @staticmethod
    def value(x, a, stream=None):
        x = _vec(x)
        call("hb2_scale", x.dtype, x.ptr, float(a), x.size(), _stream(stream))
        return x


class ElementProduct:
    @staticmethod
    def value(r, a, b, stream=None):
        r, a, b = _vec(r), _vec(a), _vec(b)
        _check_size(a.size(), b.size())
        _check_size(r.size(), a.size())
        call("hb2_element_product", r.dtype, r.ptr, a.ptr, b.ptr, r.size(), _stream(stream))
        return r


class DotProduct:
    """DotProduct<tags::B200>::value(x, y) -> host scalar (synchronises)."""

    @staticmethod
    def value(x, y, stream=None) -> float:
        x, y = _vec(x), _vec(y)
        _check_size(x.size(), y.size())
        out = ctypes.c_double()
        call("hb2_dot", x.dtype, x.ptr, y.ptr, x.size(), None, ctypes.byref(out), _stream(stream))
        return out.value


class Norm:
    """Norm<vnt_l_two, root, tags::B200>::value(x) (la/norm.hh:290-381)."""

    @staticmethod
    def value(x, root: bool = True, stream=None) -> float:
        x = _vec(x)
        out = ctypes.c_double()
        call("hb2_norm_l2", x.dtype, x.ptr, x.size(), int(bool(root)), None, ctypes.byref(out), _stream(stream))
        return out.value


def fill(x, value=0.0, stream=None):
    x = _vec(x)
    call("hb2_fill", x.dtype, x.ptr, float(value), x.size(), _stream(stream))
    return x


def copy(src, dst, stream=None):
    """copy<Tag>(source, destination) (la/algorithm.hh:50-86)."""
    src, dst = _vec(src), _vec(dst)
    _check_size(src.size(), dst.size())
    call("hb2_copy", dst.dtype, dst.ptr, src.ptr, dst.size(), _stream(stream))
    return dst


def convert(dst, src, stream=None):
    """convert<Tag>(target, source) (la/algorithm.hh:163-245)."""
    src, dst = _vec(src), _vec(dst)
    _check_size(src.size(), dst.size())
    call("hb2_convert", dst.dtype, dst.ptr, src.dtype, src.ptr, dst.size(), _stream(stream))
    return dst
