"""Generate the CSR golden fixtures from the reference implementation itself.

Runs ``oracle/_ref/honei_ref csr`` (the reference's SparseMatrixCSR constructor with
csr::blocksize 1, 2, 4 on the Q1 operator at levels 4 and 6 and 1, 3 on a skewed
5000 x 4700 matrix, and its tags::CPU Product / Defect on seeded vectors) and packs:

* ``reference_csr.npz``  -- full arrays of the level-4 cases;
* ``reference_csr.json`` -- dimensions and SHA-256 digests of the raw little-endian
  bytes of every array.

The reference sizes Aj by the matrix's nonzero count; with blocksize > 1 its tail
past Ar[rows] is never written, so only Aj[:Ar[rows]] is kept.

Usage (from the repository root, where the reference sources are available):
    make -f oracle/ref.mk -j8 && python tests/golden/make_csr_fixture.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT_DIR = os.path.join(ROOT, "tests", "golden")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "honei_ref")


def dtype_of(name: str):
    if name.endswith((".Aj", ".Ar")):
        return np.uint64
    return np.float32 if "_f32" in name else np.float64


def main() -> int:
    if not os.path.exists(REF_BIN):
        print("build the reference driver first: make -f oracle/ref.mk -j8", file=sys.stderr)
        return 1
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.check_call([REF_BIN, "csr", tmp], stdout=subprocess.DEVNULL)
        scalars = {}
        with open(os.path.join(tmp, "scalars.txt")) as f:
            for line in f:
                k, v = line.split()
                scalars[k] = int(v)
        full, digests = {}, {}
        for name in sorted(os.listdir(tmp)):
            if name == "scalars.txt":
                continue
            arr = np.fromfile(os.path.join(tmp, name), dtype=dtype_of(name))
            if name.endswith(".Aj"):
                nb = int(np.fromfile(os.path.join(tmp, name[:-3] + ".Ar"), dtype=np.uint64)[-1])
                arr = arr[:nb]
            raw = arr.tobytes()
            digests[name] = {"sha256": hashlib.sha256(raw).hexdigest(), "size": int(arr.size),
                             "dtype": np.dtype(dtype_of(name)).name}
            if name.startswith("q1_L4_"):
                full[name] = arr.copy()
    np.savez_compressed(os.path.join(OUT_DIR, "reference_csr.npz"), **full)
    with open(os.path.join(OUT_DIR, "reference_csr.json"), "w") as f:
        json.dump({"generator": "oracle/_ref/honei_ref csr (reference SparseMatrixCSR, tags::CPU)",
                   "scalars": scalars, "digests": digests}, f, indent=1, sort_keys=True)
    print(f"{len(full)} full arrays, {len(digests)} digests, {len(scalars)} scalars")
    return 0


if __name__ == "__main__":
    sys.exit(main())
