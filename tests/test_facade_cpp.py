"""The header-only C++ façade (include/hyteg_b200.hpp) compiles against the C ABI
and, on a GPU, drives a V(3,3) solve the way reference user code does."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hyteg-vara_b200")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    import sys

    sys.path.insert(0, PKG)
    import build as B

    B.build()
    out = tmp_path_factory.mktemp("facade") / "facade_gmg"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "facade_gmg.cpp"), "-L", PKG, "-lhyteg_b200",
                    f"-Wl,-rpath,{PKG}", "-o", str(out)], check=True)
    return str(out)


def test_facade_compiles_and_links(exe):
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_facade_gmg_solve(exe):
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "FACADE OK" in p.stdout
