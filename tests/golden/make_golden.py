"""Generate the committed golden fixtures from the reference implementation itself.

Runs ``oracle/_ref/honei_ref golden`` (the reference's own tags::CPU code, built
from the reference sources by ``make -f oracle/ref.mk``) and packs its outputs:

* ``reference_cpu.npz``  -- full arrays for the small cases;
* ``reference_cpu.json`` -- scalars (iteration counts, residuals, ELL dims) and
  SHA-256 digests of the raw little-endian bytes of every larger array.

Usage (from the repository root, where the reference sources are available):
    make -f oracle/ref.mk -j8 && python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT_DIR = os.path.join(ROOT, "tests", "golden")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "honei_ref")

# arrays at or below these sizes are stored in full; larger ones as digests
FULL_LIMIT = 1200 * 9


def dtype_of(name: str):
    if name.endswith((".Aj", ".Arl")):
        return np.uint64
    if "_f32" in name or name.startswith("mg32"):
        return np.float32
    return np.float64


def main() -> int:
    if not os.path.exists(REF_BIN):
        print("build the reference driver first: make -f oracle/ref.mk -j8", file=sys.stderr)
        return 1
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.check_call([REF_BIN, "golden", tmp], stdout=subprocess.DEVNULL)
        scalars = {}
        with open(os.path.join(tmp, "scalars.txt")) as f:
            for line in f:
                k, v = line.split()
                scalars[k] = float(v)
        full, digests = {}, {}
        for name in sorted(os.listdir(tmp)):
            if name == "scalars.txt":
                continue
            raw = open(os.path.join(tmp, name), "rb").read()
            arr = np.frombuffer(raw, dtype=dtype_of(name))
            digests[name] = {"sha256": hashlib.sha256(raw).hexdigest(), "size": int(arr.size),
                             "dtype": np.dtype(dtype_of(name)).name}
            if arr.size <= FULL_LIMIT:
                full[name] = arr.copy()
    np.savez_compressed(os.path.join(OUT_DIR, "reference_cpu.npz"), **full)
    with open(os.path.join(OUT_DIR, "reference_cpu.json"), "w") as f:
        json.dump({"generator": "oracle/_ref/honei_ref golden (reference tags::CPU)",
                   "scalars": scalars, "digests": digests}, f, indent=1, sort_keys=True)
    print(f"{len(full)} full arrays, {len(digests)} digests, {len(scalars)} scalars")
    return 0


if __name__ == "__main__":
    sys.exit(main())
