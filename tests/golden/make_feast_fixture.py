"""Packs the reference's MGSolverTestQuad inputs and its own result into fixtures.

Inputs: the FEAST Q1 Poisson data that the reference's math/mg_TEST.cc:398-463 reads
(testdata/poisson: A_1..A_6.ell and prol_2..prol_6.ell in the reference's binary ELL
format, rhs_6 / init_6 / sol_6 in its EXP text format).  Result: the reference's own
tags::CPU solver on that data (oracle/_ref/honei_ref mgquad: W-cycle, Jacobi 0.7,
V(4,4), coarse CG on level 1, eps 1e-8) and the restriction matrices res_2..res_6
that its MGUtil::load_data built by Transposition of each prol file, as written by
its own MatrixIO<io_formats::ELL>::write_matrix.

    python tests/golden/make_feast_fixture.py [/path/to/reference]

Writes tests/golden/feast_poisson.npz (the file arrays: each matrix's header, column
indices as uint32, values; the three vectors; the reference's solution and
restriction matrices) and
tests/golden/feast_poisson.json (iteration counts, SHA-256 of every source file).
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def read_ell(path):
    raw = open(path, "rb").read()
    head = np.frombuffer(raw[:40], dtype="<u8")
    size = int(head[0])
    aj = np.frombuffer(raw[40:40 + 8 * size], dtype="<u8")
    ax = np.frombuffer(raw[40 + 8 * size:40 + 16 * size], dtype="<f8")
    assert len(raw) == 40 + 16 * size and size == head[3] * head[4]
    return head, aj, ax


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ["HONEI_REFERENCE"]
    data = os.path.join(ref, "honei", "math", "testdata", "poisson") + "/"
    from honei_b200.io import parse_exp
    out, digests = {}, {}
    for name in [f"A_{i}.ell" for i in range(1, 7)] + [f"prol_{i}.ell" for i in range(2, 7)]:
        path = data + name
        digests[name] = hashlib.sha256(open(path, "rb").read()).hexdigest()
        head, aj, ax = read_ell(path)
        key = name[:-4]
        assert aj.max() < 2 ** 32
        out[key + ".head"] = head.astype(np.uint64)
        out[key + ".Aj"] = aj.astype(np.uint32)
        out[key + ".Ax"] = ax.copy()
    for name in ("rhs_6", "init_6", "sol_6"):
        text = open(data + name).read()
        digests[name] = hashlib.sha256(text.encode()).hexdigest()
        out[name] = parse_exp(text)
    tmp = tempfile.mkdtemp()
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "honei_ref"), "mgquad", data, tmp], check=True,
                   capture_output=True)
    out["ref_x"] = np.fromfile(os.path.join(tmp, "mgquad_x"), dtype="<f8")
    for i in range(2, 7):
        head, aj, ax = read_ell(os.path.join(tmp, f"res_{i}.ell"))
        out[f"res_{i}.head"] = head.astype(np.uint64)
        out[f"res_{i}.Aj"] = aj.astype(np.uint32)
        out[f"res_{i}.Ax"] = ax.copy()
    scalars = dict(line.split() for line in open(os.path.join(tmp, "mgquad_scalars.txt")))
    np.savez_compressed(os.path.join(HERE, "feast_poisson.npz"), **out)
    meta = {"source": "testdata/poisson of the reference (math/mg_TEST.cc:398-463)",
            "used_iters": int(scalars["used_iters"]), "used_iters_coarse": int(scalars["used_iters_coarse"]),
            "sha256": digests}
    with open(os.path.join(HERE, "feast_poisson.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print(meta["used_iters"], meta["used_iters_coarse"], os.path.getsize(os.path.join(HERE, "feast_poisson.npz")))


if __name__ == "__main__":
    main()
