"""Generate the legacy-multigrid golden fixtures from the reference implementation itself.

Packs the reference's FEAST banded Q1 test data (math/testdata/9.bin .. 1089.bin,
levels 1-5: int32 n, then 12 arrays of n doubles: DD LL LD LU DL DU UL UD UU, b, the
analytic and the reference solution) and runs ``oracle/_ref/honei_ref mglegacy`` --
the setup of math/poisson_mg_double_banded_TEST.cc and Multigrid<tags::CPU, tags::CPU,
methods::NONE, methods::JAC, methods::CYCLE::V, methods::FIXED>::value on it:

* A: the test's configuration (level 5, 16 cycles, d = b, V(2,2), factor 1, all Dirichlet);
* B: a seeded nonzero start, 30 cycles with the tolerance stop (1e-6), V(3,3), factor 0.8,
  Neumann edges (mask 2 1 2 1 2 2 1 2);
* C: smoother mode, 3 cycles, level 4;
* D: configuration A in single precision;
* E: Multigrid<..., MIXED> in the configuration of math/poisson_mg_mixed_banded_TEST.cc
  (an FP32 MGInfo with 2 cycles per outer step under FP64 defect correction);
* F: E with the adaptive coarse-grid correction (factor 0) and a seeded nonzero start.

Writes ``reference_legacy_mg.npz`` (the data arrays, shape (12, n) per level, and the
four solutions) and ``reference_legacy_mg.json`` (SHA-256 of the data files).

Usage (from the repository root, where the reference sources are available):
    make -f oracle/ref.mk -j8 && python tests/golden/make_legacy_mg_fixture.py [/path/to/reference]
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
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ["HONEI_REFERENCE"]
    data = os.path.join(ref, "honei", "math", "testdata")
    if not os.path.exists(REF_BIN):
        print("build the reference driver first: make -f oracle/ref.mk -j8", file=sys.stderr)
        return 1
    out, digests = {}, {}
    for l in range(1, 6):
        n = ((1 << l) + 1) ** 2
        raw = open(os.path.join(data, f"{n}.bin"), "rb").read()
        digests[f"{n}.bin"] = hashlib.sha256(raw).hexdigest()
        assert int(np.frombuffer(raw[:4], "<i4")[0]) == n and len(raw) == 4 + 8 * 12 * n
        out[f"bin_{n}"] = np.frombuffer(raw[4:], "<f8").reshape(12, n).copy()
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.check_call([REF_BIN, "mglegacy", data, tmp], stdout=subprocess.DEVNULL)
        for c in "ABCDEF":
            out[f"lmg_{c}.x"] = np.fromfile(os.path.join(tmp, f"lmg_{c}.x"), "<f4" if c == "D" else "<f8")
    np.savez_compressed(os.path.join(OUT_DIR, "reference_legacy_mg.npz"), **out)
    with open(os.path.join(OUT_DIR, "reference_legacy_mg.json"), "w") as f:
        json.dump({"generator": "oracle/_ref/honei_ref mglegacy (reference tags::CPU)", "sha256": digests}, f,
                  indent=1, sort_keys=True)
    print(len(out), "arrays", os.path.getsize(os.path.join(OUT_DIR, "reference_legacy_mg.npz")), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())
