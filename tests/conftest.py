import hashlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


class Golden:
    """Fixtures produced by the reference's own tags::CPU code (tests/golden/make_golden.py)."""

    def __init__(self, base="reference_cpu"):
        with open(os.path.join(GOLDEN, base + ".json")) as f:
            meta = json.load(f)
        self.scalars = meta["scalars"]
        self.digests = meta["digests"]
        self.full = dict(np.load(os.path.join(GOLDEN, base + ".npz")))

    def has(self, name):
        return name in self.digests

    def matches(self, name, arr) -> bool:
        """bit-exact comparison: full array when stored, else SHA-256 of the raw bytes"""
        d = self.digests[name]
        arr = np.ascontiguousarray(arr, dtype=np.dtype(d["dtype"]))
        if arr.size != d["size"]:
            return False
        if name in self.full:
            return np.array_equal(arr.view(np.uint8), self.full[name].view(np.uint8))
        return hashlib.sha256(arr.tobytes()).hexdigest() == d["sha256"]

    def array(self, name):
        return self.full[name]

    def scalar(self, key):
        return self.scalars[key]


@pytest.fixture(scope="session")
def golden():
    return Golden()


@pytest.fixture(scope="session")
def golden_csr():
    """reference SparseMatrixCSR fixtures (tests/golden/make_csr_fixture.py)"""
    return Golden("reference_csr")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.lib()
    return o


class Feast:
    """The reference's FEAST Q1 test data and its MGSolverTestQuad result
    (tests/golden/make_feast_fixture.py)."""

    def __init__(self):
        self.z = dict(np.load(os.path.join(GOLDEN, "feast_poisson.npz")))
        with open(os.path.join(GOLDEN, "feast_poisson.json")) as f:
            self.meta = json.load(f)

    def head(self, name):
        return [int(v) for v in self.z[name + ".head"]]

    def file_bytes(self, name) -> bytes:
        """the matrix as the reference's ELL file (five uint64, Aj as uint64, Ax)"""
        return (self.z[name + ".head"].astype("<u8").tobytes() + self.z[name + ".Aj"].astype("<u8").tobytes()
                + self.z[name + ".Ax"].astype("<f8").tobytes())

    def write(self, directory, name) -> str:
        path = os.path.join(str(directory), name + ".ell")
        with open(path, "wb") as f:
            f.write(self.file_bytes(name))
        return path

    def ell(self, oracle, name):
        return oracle.ell_from_file_arrays(self.z[name + ".head"], self.z[name + ".Aj"], self.z[name + ".Ax"])


@pytest.fixture(scope="session")
def feast():
    return Feast()
