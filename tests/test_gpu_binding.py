"""The B200 tag inside the reference tree itself: its unchanged solver templates
(MGSolver with the W-cycle of math/mg_TEST.cc:398-463 on its FEAST Q1 data,
CGSolver<Tag, NONE>) instantiated with tags::B200 (honei_b200/binding) against the
same templates with tags::CPU, in one program built from the reference's sources
(honei_b200/binding/binding.mk; prebuilt into oracle/_ref/b200/).

With the reference-order reductions the B200 run reproduces tags::CPU bit for bit
(solution, cycle and coarse-CG counts); with the library's tree-ordered reductions
the counts agree within one and the reference test's own check against sol_6
holds; a size mismatch throws VectorSizeDoesNotMatch before anything runs."""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "b200", "binding_test")


def write_feast(feast, d):
    for i in range(1, 7):
        feast.write(d, f"A_{i}")
    for i in range(2, 7):
        feast.write(d, f"prol_{i}")
    for name in ("rhs_6", "init_6", "sol_6"):
        (d / name).write_text("# " + name + "\n" + "".join("%.17g\n" % v for v in feast.z[name]))


def test_reference_templates_with_the_b200_tag(feast, tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("binding not built (make -f honei_b200/binding/binding.mk REF=<reference>)")
    data = tmp_path / "feast"
    data.mkdir()
    write_feast(feast, data)
    rc = tmp_path / "honeirc"
    rc.write_text("log::categories = none\nlog::output = /dev/null\n")
    out = subprocess.run([BIN, str(data) + "/"], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, HONEI_CONFIG=str(rc)))
    assert out.returncode == 0, out.stderr[-2000:]
    line = next(l for l in out.stdout.splitlines() if l.startswith("RESULT "))
    r = json.loads(line[len("RESULT "):])
    assert r["feast_cpu_iters"] == feast.meta["used_iters"] and r["feast_cpu_coarse"] == feast.meta["used_iters_coarse"]
    assert r["feast_exact_same_bits"], r
    assert (r["feast_exact_iters"], r["feast_exact_coarse"]) == (r["feast_cpu_iters"], r["feast_cpu_coarse"])
    assert abs(r["feast_tree_iters"] - r["feast_cpu_iters"]) <= 1 and r["feast_tree_test_ok"] and r["feast_cpu_test_ok"]
    assert r["feast_tree_max_diff"] < 1e-8
    assert r["cg_exact_same_bits"] and r["cg_exact_iters"] == r["cg_cpu_iters"]
    assert abs(r["cg_tree_iters"] - r["cg_cpu_iters"]) <= 1 and r["cg_tree_max_diff"] < 1e-6
    assert r["size_check_throws"]
