"""The C++ operator and solver templates of the B200 tag (include/honei_b200.hh):
tests/cpp/operators_test.cc built with g++ against libhonei_b200.so, the oracle's C
library and the CUDA runtime, and run on the GPU against the oracle."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "operators_test.cc")
CUDA = "/usr/local/cuda"
LIB_DIR = os.path.join(ROOT, "honei_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")


def build(out_dir) -> str:
    for path in (os.path.join(LIB_DIR, "libhonei_b200.so"), os.path.join(ORACLE_DIR, "liboracle.so")):
        if not os.path.exists(path):
            pytest.skip(f"{os.path.basename(path)} not built (python -c 'import __graft_entry__ as g; g.build()')")
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = os.path.join(str(out_dir), "operators_test")
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-Wall", "-Wextra",
           "-I", os.path.join(ROOT, "include"), "-I", ORACLE_DIR, "-I", os.path.join(CUDA, "include"),
           SRC, "-o", exe,
           "-L", LIB_DIR, "-lhonei_b200", "-L", ORACLE_DIR, "-loracle", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{LIB_DIR}:{ORACLE_DIR}:{os.path.join(CUDA, 'lib64')}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    assert "warning" not in res.stderr, res.stderr
    return exe


def test_cpp_layer_builds(tmp_path):
    """The header compiles warning-free as C++17 and links against the library."""
    build(tmp_path)


@pytest.mark.gpu
def test_cpp_layer_matches_oracle(tmp_path):
    exe = build(tmp_path)
    res = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "14 tests, 0 failed" in res.stdout, res.stdout
