"""honei_b200 -- B200 (sm_100a) backend of HONEI's sparse Poisson solver path.

Python mirror of the reference's tag-dispatched operator API over the C ABI in
include/honei_b200.h (libhonei_b200.so).  There is no CPU fallback: the first
operator call without the built library raises ImportError.
"""
from ._lib import DeviceTimeout, HoneiError, NotFinite, VectorSizeDoesNotMatch, launch_count
from .io import MatrixIO, VectorIO, io_formats
from .la import (BandedMatrixQx, Defect, DenseVector, Difference, DotProduct, ElementProduct, Norm, Product, Scale,
                 ScaledSum, SparseMatrixCSR, SparseMatrixELL, Sum, convert, copy, fill, tags)
from .solvers import (HB2_BICGSTAB_VAR, HB2_CG_SMOOTHER, HB2_CG_VAR, BatchedPoissonSolver, BiCGStabSolver, CGSmoother,
                      CGSolver, IRSolver, KrylovSolver, MGData, MGSolver, Multigrid, Prolongation, Restriction,
                      RISmoother, batch_params, methods, mg_info, mg_params)

__all__ = [
    "BandedMatrixQx", "BatchedPoissonSolver", "BiCGStabSolver", "CGSmoother", "CGSolver", "HB2_BICGSTAB_VAR",
    "HB2_CG_SMOOTHER", "HB2_CG_VAR", "KrylovSolver", "Defect", "DenseVector", "DeviceTimeout", "Difference", "DotProduct",
    "ElementProduct", "HoneiError", "MatrixIO", "VectorIO", "io_formats", "IRSolver", "MGData", "MGSolver", "Norm", "NotFinite", "Product",
    "Prolongation", "RISmoother", "Restriction", "Scale", "ScaledSum", "SparseMatrixCSR", "SparseMatrixELL", "Sum",
    "VectorSizeDoesNotMatch", "batch_params", "convert", "copy", "fill", "launch_count", "methods", "mg_info", "mg_params", "Multigrid", "tags",
]
