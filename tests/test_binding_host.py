"""The B200 tag binding (honei_b200/binding) compiles against the reference tree's
own headers -- C++98 as the tree is, warnings as errors -- with the tree's
tags.hh carrying the one added tag value (the overlay binding.mk makes).  Needs the
reference checkout (HONEI_REFERENCE); compiles only, runs nothing."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("HONEI_REFERENCE", "")


@pytest.mark.skipif(not (REF and os.path.isdir(os.path.join(REF, "honei"))), reason="reference sources not present")
def test_binding_compiles_warning_free(tmp_path):
    ovl = tmp_path / "overlay" / "honei" / "util"
    ovl.mkdir(parents=True)
    src = open(os.path.join(REF, "honei", "util", "tags.hh")).read()
    lines = []
    for line in src.splitlines():
        if line.strip() == "tv_none":
            lines.append(line.replace("tv_none", "tv_b200,"))
        lines.append(line)
    (ovl / "tags.hh").write_text("\n".join(lines) + "\n")
    for f in ("honei_b200/binding/b200_backend.cc", "tests/cpp/binding_test.cc"):
        cmd = ["g++", "-std=gnu++98", "-fsyntax-only", "-DHONEI_SSE", "-fpermissive", "-Wall", "-Wextra", "-Werror",
               "-isystem", str(tmp_path / "overlay"), "-isystem", REF, "-isystem", "/usr/local/cuda/include",
               "-Iinclude", "-Ihonei_b200/binding", f'-DHONEI_SOURCEDIR="{REF}"', f]
        out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
        assert out.returncode == 0 and not out.stderr.strip(), out.stderr[-3000:]
