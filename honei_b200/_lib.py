"""ctypes binding of libhonei_b200.so (the C ABI declared in include/honei_b200.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libhonei_b200.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "honei_b200.h")

HB2_F64, HB2_F32 = 0, 1
HB2_OK = 0
HB2_ERR_ARG = -1
HB2_ERR_SIZE = -2
HB2_ERR_CUDA = -3
HB2_ERR_NOMEM = -4
HB2_ERR_TIMEOUT = -5
HB2_ERR_UNSUPPORTED = -6
HB2_ERR_NOT_FINITE = -7


class HoneiError(RuntimeError):
    """InternalError of the reference (util/exception.hh): a backend failure."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class VectorSizeDoesNotMatch(HoneiError):
    """la/vector_error.hh: raised before anything is launched."""


class DeviceTimeout(HoneiError):
    """A bounded device-side wait expired (the kernel returned instead of hanging)."""


class NotFinite(HoneiError):
    """A solver produced a NaN/Inf residual norm."""


_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32
_int = ctypes.c_int
_dbl = ctypes.c_double
_vp = ctypes.c_void_p
_pvp = ctypes.POINTER(ctypes.c_void_p)
_pu64 = ctypes.POINTER(ctypes.c_uint64)
_pdbl = ctypes.POINTER(ctypes.c_double)


class MgParams(ctypes.Structure):
    """hb2_mg_params"""
    _fields_ = [("n_pre_smooth", _u64), ("n_post_smooth", _u64), ("max_iters", _u64),
                ("max_iters_coarse", _u64), ("eps_relative", _dbl), ("coarse_eps", _dbl), ("omega", _dbl),
                ("coarse_exact", _int), ("no_fused_levels", _int), ("coarse_fp64", _int), ("cycle", _int)]


class MGInfoParams(ctypes.Structure):
    """hb2_lmg_params (MGInfo, math/multigrid.hh:65-149)"""
    _fields_ = [("n_max_iter", _u64), ("initial_zero", _int), ("convergence_check", _int), ("is_smoother", _int),
                ("tolerance", _dbl), ("n_pre_smooth", _u64), ("adapt_correction_factor", _dbl), ("omega", _dbl),
                ("macro_border_mask", _u64 * 8), ("adaptive", _int)]


class BatchParams(ctypes.Structure):
    """hb2_batch_params"""
    _fields_ = [("max_iters", _u64), ("eps_relative", _dbl), ("n_pre_smooth", _u64), ("n_post_smooth", _u64),
                ("max_iters_coarse", _u64), ("coarse_eps", _dbl), ("omega", _dbl)]


# name -> (restype, argtypes)
SIGNATURES = {
    "hb2_last_error": (ctypes.c_char_p, []),
    "hb2_version": (ctypes.c_char_p, []),
    "hb2_launch_count": (_u64, []),
    "hb2_workspace_count": (_u64, []),
    "hb2_ell_create": (_int, [_pvp, _int, _u64, _u64, _u64, _u64, _u64, _vp, _vp, _vp, _int, _vp]),
    "hb2_ell_create_q1": (_int, [_pvp, _int, ctypes.c_uint, _dbl, _vp]),
    "hb2_ell_create_transfer": (_int, [_pvp, _pvp, _int, ctypes.c_uint, _vp]),
    "hb2_ell_convert": (_int, [_pvp, _vp, _int, _vp]),
    "hb2_ell_destroy": (_int, [_vp]),
    "hb2_ell_info": (_int, [_vp, _pu64, _pu64, _pu64, _pu64, _pu64, _pu64]),
    "hb2_ell_export": (_int, [_vp, _vp, _vp, _vp]),
    "hb2_ell_layout": (_int, [_vp, ctypes.POINTER(_int), ctypes.POINTER(_u32), ctypes.POINTER(_u32)]),
    "hb2_ell_layout_variant": (_int, [_vp, _int, ctypes.POINTER(_int), ctypes.POINTER(_int), ctypes.POINTER(_int)]),
    "hb2_ell_launch_shape": (_int, [_vp, _int, ctypes.POINTER(_int), ctypes.POINTER(_int)]),
    "hb2_ell_read": (_int, [_pvp, ctypes.c_char_p, _int, _vp]),
    "hb2_ell_write": (_int, [_vp, ctypes.c_char_p]),
    "hb2_ell_transpose": (_int, [_pvp, _vp, _vp]),
    "hb2_ell_create_bf16": (_int, [_pvp, _vp, _int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                   _vp]),
    "hb2_lmg_create": (_int, [_pvp, ctypes.c_uint, ctypes.c_uint, _vp, _vp, _vp]),
    "hb2_lmg_destroy": (_int, [_vp]),
    "hb2_lmg_solve": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hb2_lmg_solve_mixed": (_int, [_vp, _vp, _vp, _vp, _u64, _vp, _vp, _vp, _vp]),
    "hb2_krylov_create": (_int, [_pvp, _int, _vp, _vp, _vp, _u64, _dbl, _vp]),
    "hb2_krylov_destroy": (_int, [_vp]),
    "hb2_krylov_solve": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hb2_csr_create": (_int, [_pvp, _int, _u64, _u64, _u64, _vp, _vp, _vp, _int, _vp]),
    "hb2_csr_from_ell": (_int, [_pvp, _vp, _u64, _vp]),
    "hb2_csr_destroy": (_int, [_vp]),
    "hb2_csr_info": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hb2_csr_export": (_int, [_vp, _vp, _vp, _vp]),
    "hb2_csr_layout": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "hb2_product_csr": (_int, [_vp, _vp, _vp, _vp]),
    "hb2_defect_csr": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "hb2_q1_create": (_int, [_pvp, _int, _u64, _vp, _int, _vp]),
    "hb2_q1_create_poisson": (_int, [_pvp, _int, ctypes.c_uint, _dbl, _vp]),
    "hb2_q1_destroy": (_int, [_vp]),
    "hb2_product_ell": (_int, [_vp, _vp, _vp, _vp]),
    "hb2_defect_ell": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hb2_defect_ell_noalloc": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hb2_product_dot_ell": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "hb2_product_add_ell": (_int, [_vp, _vp, _vp, _vp]),
    "hb2_product_q1": (_int, [_vp, _vp, _vp, _vp]),
    "hb2_defect_q1": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "hb2_scaled_sum": (_int, [_int, _vp, _vp, _dbl, _u64, _vp]),
    "hb2_scaled_sum3": (_int, [_int, _vp, _vp, _vp, _dbl, _u64, _vp]),
    "hb2_sum": (_int, [_int, _vp, _vp, _u64, _vp]),
    "hb2_difference": (_int, [_int, _vp, _vp, _u64, _vp]),
    "hb2_difference3": (_int, [_int, _vp, _vp, _vp, _u64, _vp]),
    "hb2_scale": (_int, [_int, _vp, _dbl, _u64, _vp]),
    "hb2_element_product": (_int, [_int, _vp, _vp, _vp, _u64, _vp]),
    "hb2_fill": (_int, [_int, _vp, _dbl, _u64, _vp]),
    "hb2_copy": (_int, [_int, _vp, _vp, _u64, _vp]),
    "hb2_convert": (_int, [_int, _vp, _int, _vp, _u64, _vp]),
    "hb2_dot": (_int, [_int, _vp, _vp, _u64, _vp, _vp, _vp]),
    "hb2_norm_l2": (_int, [_int, _vp, _u64, _int, _vp, _vp, _vp]),
    "hb2_dot_ordered": (_int, [_int, _vp, _vp, _u64, _int, _vp, _vp, _vp]),
    "hb2_prolongation": (_int, [_int, _vp, _u64, _vp, _u64, _vp, _vp]),
    "hb2_restriction": (_int, [_int, _vp, _u64, _vp, _u64, _vp, _vp]),
    "hb2_jacobi_ell": (_int, [_vp, _vp, _vp, _vp, _vp, _u64, _vp]),
    "hb2_jacobi_precon": (_int, [_vp, _dbl, _vp, _vp]),
    "hb2_jacobi_sweep_ell": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hb2_cg_solve": (_int, [_vp, _vp, _vp, _u64, _dbl, _pu64, _pdbl, _vp]),
    "hb2_mg_create": (_int, [_pvp, _u32, _vp, _vp, _vp, ctypes.POINTER(MgParams), _vp]),
    "hb2_mg_create_q1": (_int, [_pvp, _int, ctypes.c_uint, ctypes.c_uint, _dbl, ctypes.POINTER(MgParams), _vp]),
    "hb2_mg_destroy": (_int, [_vp]),
    "hb2_mg_solve": (_int, [_vp, _vp, _vp, _pdbl, _vp]),
    "hb2_mg_cycle": (_int, [_vp, _vp, _vp, _vp]),
    "hb2_ir_solve": (_int, [_vp, _vp, _vp, _vp, _dbl, _u64, _int, _pdbl, _vp]),
    "hb2_batch_create_q1": (_int, [_pvp, _u32, _vp, _vp, ctypes.c_uint, ctypes.POINTER(BatchParams), _vp]),
    "hb2_batch_destroy": (_int, [_vp]),
    "hb2_batch_info": (_int, [_vp, ctypes.POINTER(_u32), _pu64, _pu64]),
    "hb2_batch_copy": (_int, [_vp, _u32, _int, _vp, _vp]),
    "hb2_batch_start": (_int, [_vp, _u32, _dbl, _int, _vp]),
    "hb2_batch_step": (_int, [_vp, _u32, _vp, _vp]),
    "hb2_batch_solve": (_int, [_vp, _int, _pu64, _vp]),
    "hb2_batch_result": (_int, [_vp, _u32, _u32, _pu64, _pdbl]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load the in-tree library (built by ``python -m honei_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m honei_b200.build` "
                              "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int, what: str = "") -> None:
    if status == HB2_OK:
        return
    msg = load().hb2_last_error().decode(errors="replace")
    if what:
        msg = f"{what}: {msg}"
    if status == HB2_ERR_SIZE:
        raise VectorSizeDoesNotMatch(status, msg)
    if status == HB2_ERR_TIMEOUT:
        raise DeviceTimeout(status, msg)
    if status == HB2_ERR_NOT_FINITE:
        raise NotFinite(status, msg)
    raise HoneiError(status, msg)


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)


def launch_count() -> int:
    return int(load().hb2_launch_count())
