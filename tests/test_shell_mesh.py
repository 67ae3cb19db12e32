"""The product's spherical-shell generator (hyteg-vara_b200/csrc/topology.cpp
meshSphericalShell, behind hyb_storage_create_spherical_shell) against the reference's own
MeshInfo::meshSphericalShell (src/hyteg/mesh/MeshGenSphericalShell.cpp:577-900,
SHELLMESH_CLASSIC), compiled unchanged by tests/golden/make_shell_mesh_golden.py, which wrote
tests/golden/shell_mesh_reference.npz: the same vertex ids (coordinates to 1e-15), the same
cells in the same order with the same vertex order -- so config 5 and the curved-shell runs
use the reference's mesh. The generator is compiled here with g++ (it has no device code)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "hyteg-vara_b200", "csrc")
GOLD = np.load(os.path.join(ROOT, "tests", "golden", "shell_mesh_reference.npz"))

MAIN = r"""
#include "topology.hpp"
#include <cstdio>
#include <cstdlib>
int main( int argc, char** argv )
{
   std::vector< std::array< double, 3 > > V;
   std::vector< std::array< int, 4 > >    T;
   hyb::meshSphericalShell( atoi( argv[1] ), atoi( argv[2] ), atof( argv[3] ), atof( argv[4] ), V, T );
   printf( "%zu %zu\n", V.size(), T.size() );
   for ( auto& v : V ) printf( "%.17g %.17g %.17g\n", v[0], v[1], v[2] );
   for ( auto& t : T ) printf( "%d %d %d %d\n", t[0], t[1], t[2], t[3] );
}
"""


@pytest.fixture(scope="module")
def generator(tmp_path_factory):
    d = tmp_path_factory.mktemp("shell")
    src, exe = d / "m.cpp", d / "m"
    src.write_text(MAIN)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, str(src), os.path.join(CSRC, "topology.cpp"), "-o", str(exe)],
                   check=True)

    def run(ntan, nrad, rmin=0.55, rmax=1.0):
        lines = subprocess.run([str(exe), str(ntan), str(nrad), repr(rmin), repr(rmax)], check=True, capture_output=True,
                               text=True).stdout.split("\n")
        nv, nt = map(int, lines[0].split())
        V = np.array([[float(x) for x in l.split()] for l in lines[1:1 + nv]])
        T = np.array([[int(x) for x in l.split()] for l in lines[1 + nv:1 + nv + nt]], dtype=np.int64)
        return V, T

    return run


@pytest.mark.parametrize("ntan,nrad", [(3, 2), (5, 3), (5, 4)])
def test_shell_mesh_is_the_references(generator, ntan, nrad):
    V, T = generator(ntan, nrad)
    Vr, Tr = GOLD[f"ntan{ntan}_nrad{nrad}_coords"], GOLD[f"ntan{ntan}_nrad{nrad}_tets"]
    assert V.shape == Vr.shape and T.shape == Tr.shape
    assert np.abs(V - Vr).max() <= 1e-15
    assert np.array_equal(T, Tr)


def test_shell_mesh_counts_and_radii(generator):
    """(10 (ntan-1)^2 + 2) nrad vertices on the nrad radii, 60 (ntan-1)^2 (nrad-1) cells, all
    positively or negatively oriented but none degenerate."""
    V, T = generator(5, 4)
    assert len(V) == (10 * 16 + 2) * 4 and len(T) == 60 * 16 * 3
    r = np.linalg.norm(V, axis=1)
    assert np.allclose(np.sort(np.unique(np.round(r, 12))), [0.55, 0.7, 0.85, 1.0])
    X = V[T]
    vol = np.abs(np.linalg.det(X[:, 1:] - X[:, :1])) / 6
    assert vol.min() > 1e-4


def test_shell_mesh_rejects_classic_incompatible_ntan(generator):
    with pytest.raises(subprocess.CalledProcessError):
        generator(4, 2)
