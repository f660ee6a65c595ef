"""bench.py's host-side helpers: the algorithmic byte model of an MG solve, the kernel
variant names and their committed ncu traffic, the strict-JSON handling of a diverged
solve's numbers, and the batched workload's shape."""
import json
import math
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_mg_solve_bytes_counts_every_pass():
    """Levels 3..4, one cycle, V(4,4): sweeps, defect, transfers, the coarse solve and
    the convergence defects, each vector / matrix entry once per pass."""
    rb = {"A": 1, "R": 27, "P": 12}
    s = 8
    nf, nc = 17 ** 2, 9 ** 2
    level4 = 8 * nf * (1 + 4 * s) + nf * (1 + 3 * s) + nc * (27 + 2 * s) + nf * s + nf * (12 + 2 * s) + nc * s
    coarse = nc * (1 + 2 * s)
    conv = nf * (1 + 3 * s)
    want = (level4 + coarse + conv) + conv
    assert bench.mg_solve_bytes(4, 1, lambda l, w: rb[w], min_level=3) == want
    # the Q1 transfer kernels read no matrix: fewer bytes, by exactly the matrix bytes
    rb0 = {"A": 1, "R": 0, "P": 0}
    assert bench.mg_solve_bytes(4, 1, lambda l, w: rb0[w], min_level=3) == want - nc * 27 - nf * 12


def test_variant_names_and_committed_traffic():
    assert bench.variant_name(2, 2, False) == "pattern2"
    assert bench.variant_name(2, 1, True) == "patternwin1"
    assert bench.variant_name(2, 4, 2) == "q1stencil4"
    assert bench.variant_name(2, 2, 3) == "q1gather2"
    assert bench.variant_name(2, 2, 4) == "q1pair"
    assert bench.variant_name(2, 4, 5) == "q1strip4"
    assert bench.variant_name(3, 1, 0) == "bf16r1"
    assert bench.variant_name(1, 4, False) == "force4"
    assert bench.variant_name(0, 2, False) == "plain"
    for v in ("pattern1", "pattern2", "pattern4", "patternwin1", "patternwin2"):
        t = bench.load_traffic(f"{v}:jacobi:L10")
        # DRAM bytes of one level-10 sweep: about the 25 B/row the kernel must read
        assert t is not None and 25 * 1_050_625 <= t <= 25.1 * 1_050_625
    assert bench.load_traffic("force8:jacobi:L10") is None
    # the level-11 kernels the bench reports
    for key in ("q1gather1:jacobi:L11", "plain:spmv:L11", "plain:defect:L11", "plain:jacobi:L11:coefficients",
                "bf16r2:jacobi:L11:coefficients-compensated"):
        assert bench.load_traffic(key) is not None, key


def test_error_bound_from_residuals():
    """the Q1 operator's smallest eigenvalue (smooth interior mode) and the bound on
    the distance of two solutions from their residuals"""
    import numpy as np
    lam = bench.q1_lambda_min(11)
    assert abs(lam - 4.706e-6) < 1e-8
    keep = {"xir": np.ones(4) * 1.0 + 1e-9, "x64": np.ones(4), "b": np.ones(4) * 2.0, "relres_mixed": 1e-11}
    e = bench.solution_errors(11, keep, np.ones(4), 2e-11, "test")
    assert abs(e["mixed_rel_error_vs_reference_fp64"] - 1e-9) < 1e-15
    assert e["fp64_gpu_rel_error_vs_reference_fp64"] == 0.0
    assert abs(e["mixed_error_bound_from_residuals"] - 3e-11 * 4.0 / (lam * 2.0)) < 1e-12


def test_diverged_numbers_stay_strict_json():
    line = {"a": bench.finite_or_text(1.5), "b": bench.finite_or_text(float("inf")),
            "c": bench.finite_or_text(float("nan"))}
    text = json.dumps(line)

    def reject(name):
        raise ValueError(name)

    back = json.loads(text, parse_constant=reject)
    assert back == {"a": 1.5, "b": "inf", "c": "nan"}
    assert math.isfinite(back["a"])


def test_batched_workload_shape():
    w = bench.batch_workload(7)
    assert len(w) == 512
    assert sum(1 for _, k in w if k == 8) == 128 and all(k in (1, 8) for _, k in w)
    assert all(4 <= l <= 9 for l, _ in w)
    assert bench.batch_workload(7) == w


def test_percentile():
    assert bench.percentile([1.0, 2.0, 3.0, 4.0], 50) in (2.0, 2.5, 3.0)
    assert bench.percentile([5.0], 99) == 5.0
