"""Generate the Krylov-solver golden fixtures from the reference implementation itself.

Runs ``oracle/_ref/honei_ref krylov`` -- the reference's CGSolver<tags::CPU,
methods::VAR>, BiCGStabSolver<tags::CPU, methods::VAR> and CGSmoother on the Q1
operator at levels 5 and 6 (b = A u, x0 = 0, eps 1e-8, at most 1000 iterations),
preconditioned by the Jacobi vector 1 / diag(A) or by the ELL matrix
P = 2 D^-1 - D^-1 A D^-1 -- and packs:

* ``reference_krylov.npz``  -- full arrays of the level-5 cases;
* ``reference_krylov.json`` -- iteration counts, relative residuals and SHA-256
  digests of every array.

Usage (from the repository root, where the reference sources are available):
    make -f oracle/ref.mk -j8 && python tests/golden/make_krylov_fixture.py
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


def main() -> int:
    if not os.path.exists(REF_BIN):
        print("build the reference driver first: make -f oracle/ref.mk -j8", file=sys.stderr)
        return 1
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.check_call([REF_BIN, "krylov", tmp], stdout=subprocess.DEVNULL)
        scalars = {}
        with open(os.path.join(tmp, "scalars.txt")) as f:
            for line in f:
                k, v = line.split()
                scalars[k] = float(v)
        full, digests = {}, {}
        for name in sorted(os.listdir(tmp)):
            if name == "scalars.txt":
                continue
            dt = np.uint64 if name.endswith((".Aj", ".Arl")) else np.float64
            arr = np.fromfile(os.path.join(tmp, name), dtype=dt)
            digests[name] = {"sha256": hashlib.sha256(arr.tobytes()).hexdigest(), "size": int(arr.size),
                             "dtype": np.dtype(dt).name}
            if name.startswith("kr_L5.") and ".Pn." not in name:
                full[name] = arr.copy()
    np.savez_compressed(os.path.join(OUT_DIR, "reference_krylov.npz"), **full)
    with open(os.path.join(OUT_DIR, "reference_krylov.json"), "w") as f:
        json.dump({"generator": "oracle/_ref/honei_ref krylov (reference tags::CPU)",
                   "scalars": scalars, "digests": digests}, f, indent=1, sort_keys=True)
    print(f"{len(full)} full arrays, {len(digests)} digests, {len(scalars)} scalars")
    return 0


if __name__ == "__main__":
    sys.exit(main())
