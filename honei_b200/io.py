"""File formats of the reference (math/matrix_io.hh, math/vector_io.hh).

MatrixIO.read_matrix / write_matrix: MatrixIO<io_formats::ELL> -- the binary ELL
file (five uint64: size, rows, columns, stride, num_cols_per_row; size uint64 column
indices; size doubles), read straight into the device layout (hb2_ell_read).
VectorIO: VectorIO<io_formats::EXP> (text, one number per line, lines with '#'
skipped; math/vector_io.hh:55-110) and VectorIO<io_formats::DV> (binary: uint64
size, then the doubles; math/vector_io.hh:205-250).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from ._lib import call
from .la import DenseVector, SparseMatrixELL, _stream, dtype_code


class io_formats:
    ELL = "ell"
    EXP = "exp"
    DV = "dv"


class MatrixIO:
    @staticmethod
    def read_matrix(path, dtype=torch.float64, stream=None) -> SparseMatrixELL:
        h = ctypes.c_void_p()
        call("hb2_ell_read", ctypes.byref(h), os.fsencode(path), dtype_code(dtype), _stream(stream))
        return SparseMatrixELL._from_handle(h, dtype)

    @staticmethod
    def write_matrix(path, A: SparseMatrixELL):
        call("hb2_ell_write", A.handle, os.fsencode(path))


def parse_exp(text: str) -> np.ndarray:
    """VectorIO<EXP>::read_vector: getline until end of file; a line containing '#'
    is skipped; a line that ends the file without a newline is dropped; every other
    line is atof of its text after leading blanks (an empty line reads as 0)."""
    lines = text.split("\n")[:-1]
    vals = []
    for line in lines:
        if "#" in line:
            continue
        s = line.lstrip(" ")
        try:
            vals.append(float(s.split()[0]) if s.split() else 0.0)
        except ValueError:
            vals.append(0.0)
    return np.array(vals, dtype=np.float64)


class VectorIO:
    @staticmethod
    def read_vector(path, fmt=io_formats.EXP, dtype=torch.float64, device="cuda") -> DenseVector:
        if fmt == io_formats.EXP:
            with open(path) as f:
                v = parse_exp(f.read())
        elif fmt == io_formats.DV:
            with open(path, "rb") as f:
                n = int(np.frombuffer(f.read(8), dtype="<u8")[0])
                v = np.frombuffer(f.read(8 * n), dtype="<f8")
                if v.size != n:
                    raise IOError(f"{path}: short DV file")
        else:
            raise ValueError(f"unknown vector format {fmt!r}")
        return DenseVector(torch.from_numpy(v.copy()).to(dtype), device=device)

    @staticmethod
    def write_vector(path, v, fmt=io_formats.DV):
        """VectorIO<DV>::write_vector (values written as doubles)."""
        if fmt != io_formats.DV:
            raise ValueError("the reference writes vectors in the DV format only")
        a = (v.elements if hasattr(v, "elements") else v).detach().to(torch.float64).cpu().numpy()
        with open(path, "wb") as f:
            f.write(np.array([a.size], dtype="<u8").tobytes())
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
