"""The header-only ddj layer (include/gtsc/ddj.hpp): reference-style C++ client code compiles
against it (CPU) and runs correctly on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gputimeseriescompressionoptimizer_b200")


def build(tmp_path):
    exe = str(tmp_path / "ddj_shim_test")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "ddj_shim_test.cpp"), "-o", exe, "-L", PKG, "-lgtsc",
                    f"-Wl,-rpath,{PKG}"], check=True)
    return exe


def test_ddj_shim_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_ddj_shim_runs(tmp_path):
    r = subprocess.run([build(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "all checks passed" in r.stdout
