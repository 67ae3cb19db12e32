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


@pytest.fixture(scope="module")
def exe_smoothers(tmp_path_factory):
    import sys

    sys.path.insert(0, PKG)
    import build as B

    B.build()
    out = tmp_path_factory.mktemp("facade") / "facade_smoothers"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "facade_smoothers.cpp"), "-L", PKG, "-lhyteg_b200",
                    f"-Wl,-rpath,{PKG}", "-o", str(out)], check=True)
    return str(out)


def test_facade_smoothers_compile(exe_smoothers):
    assert os.path.exists(exe_smoothers)


@pytest.mark.gpu
def test_facade_smoothers_and_gmsh(exe_smoothers, tmp_path, write_gmsh):
    """W-cycles with symmetric SOR, Chebyshev with the estimated spectral radius, full
    multigrid, and a reference test mesh (regular_octahedron_8el) read from a Gmsh file."""
    import numpy as np

    g = np.load(os.path.join(ROOT, "tests", "golden", "reference_meshes.npz"))
    msh = tmp_path / "octahedron.msh"
    write_gmsh(msh, g["regular_octahedron_8el_coords"], g["regular_octahedron_8el_tets"], seed=5)
    p = subprocess.run([exe_smoothers, str(msh)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "FACADE SMOOTHERS OK" in p.stdout
