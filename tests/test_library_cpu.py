"""CPU-side checks of the product library: it builds for sm_100a, loads, and exports
every entry point include/hyteg_b200.h declares; the host topology (multicolour
labelling) is valid on the reference's meshes. No GPU compute is called here."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hyteg-vara_b200")
HEADER = os.path.join(ROOT, "include", "hyteg_b200.h")


def header_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(hyb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    sys.path.insert(0, PKG)
    import build as B

    B.build()
    import hyteg_b200 as H

    return H.load()


def test_library_exports_every_declared_symbol(lib):
    import hyteg_b200 as H

    syms = header_symbols()
    assert syms, "no declarations parsed"
    assert sorted(H.SYMBOLS) == syms
    for s in syms:
        assert hasattr(lib, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(PKG, "libhyteg_b200.so")], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (hyb_[a-z0-9_]+)", out))
    assert set(syms) <= exported


def test_library_is_built_for_sm100a(lib):
    import build as B

    assert "arch=compute_100a,code=sm_100a" in B.FLAGS
    assert B.up_to_date()


def test_last_error_without_device(lib):
    # no compute call: only the error channel is exercised
    assert isinstance(lib.hyb_last_error(), bytes)


TOPO_CHECK = r"""
#include "topology.hpp"
#include <cstdio>
#include <cstdlib>
#include <vector>
using namespace hyb;
int main( int argc, char** argv )
{
   // stdin: nv nt, coords, tets; stdout: colours, valid, nE, nF, then labels
   long nv, nt;
   if ( scanf( "%ld %ld", &nv, &nt ) != 2 ) return 2;
   std::vector< std::array< double, 3 > > V( nv );
   std::vector< std::array< int, 4 > > T( nt );
   for ( auto& v : V ) if ( scanf( "%lf %lf %lf", &v[0], &v[1], &v[2] ) != 3 ) return 2;
   for ( auto& t : T ) if ( scanf( "%d %d %d %d", &t[0], &t[1], &t[2], &t[3] ) != 4 ) return 2;
   Topology tp;
   tp.build( V, T );
   tp.computeColouring();
   printf( "%d %d %zu %zu\n", tp.colours, tp.colouringValid() ? 1 : 0, tp.E.size(), tp.F.size() );
   for ( int l : tp.labels ) printf( "%d ", l );
   printf( "\n" );
   return 0;
}
"""


@pytest.fixture(scope="module")
def topo_exe(tmp_path_factory):
    d = tmp_path_factory.mktemp("topo")
    src = d / "topo_check.cpp"
    src.write_text(TOPO_CHECK)
    exe = d / "topo_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(PKG, "csrc"), str(src),
                    os.path.join(PKG, "csrc", "topology.cpp"), "-o", str(exe)], check=True)
    return str(exe)


def run_topo(exe, coords, tets):
    inp = f"{len(coords)} {len(tets)}\n" + "\n".join(" ".join(map(repr, map(float, c))) for c in coords) + "\n" + \
        "\n".join(" ".join(map(str, t)) for t in tets) + "\n"
    out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    m, valid, ne, nf = map(int, out[0].split())
    labels = np.array(list(map(int, out[1].split())))
    return m, valid, ne, nf, labels


def colouring_separates_couplings(oracle_mod, coords, tets, labels, m, level=2):
    """Every pair of micro-vertices coupled by the operator gets different colours."""
    O = oracle_mod
    o = O.Oracle(coords, tets, level)
    n = o.n(level)
    xyz = o.coords_of(level)
    # colour of every DoF from its barycentric key in its first cell
    col = np.full(n, -1)
    N = 1 << level
    for c, t in enumerate(tets):
        cm = o.closure_map(level, c)
        idx = 0
        for z in range(N + 1):
            for y in range(N + 1 - z):
                for x in range(N + 1 - y - z):
                    b = (N - x - y - z, x, y, z)
                    col[cm[idx]] = sum(labels[t[k]] * b[k] for k in range(4)) % m
                    idx += 1
    # couplings from the operator: A e_j has nonzeros at the coupled rows
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        y = o.apply(e, level, flag=O.ALL)
        nz = np.nonzero(np.abs(y) > 1e-14)[0]
        for i in nz:
            if i != j:
                assert col[i] != col[j], (i, j)
    return True


@pytest.mark.parametrize("mesh", ["cube1", "cube2", "octahedron", "pyramid"])
def test_multicolour_labelling_is_valid(topo_exe, oracle_mod, mesh):
    O = oracle_mod
    if mesh == "cube1":
        c, t = O.mesh_cuboid(1, 1, 1)
    elif mesh == "cube2":
        c, t = O.mesh_cuboid(2, 2, 2)
    else:
        g = np.load(os.path.join(ROOT, "tests", "golden", "reference_meshes.npz"))
        name = "regular_octahedron_8el" if mesh == "octahedron" else "pyramid_4el"
        c, t = g[name + "_coords"], g[name + "_tets"]
    m, valid, ne, nf, labels = run_topo(topo_exe, c, t)
    assert valid == 1 and m >= 4
    assert colouring_separates_couplings(O, c, t, labels, m, level=2)


def test_topology_counts_match_oracle(topo_exe, oracle_mod):
    O = oracle_mod
    c, t = O.mesh_cuboid(2, 2, 2)
    m, valid, ne, nf, labels = run_topo(topo_exe, c, t)
    o = O.Oracle(c, t, 0)
    assert ne == o.num_prims(1) and nf == o.num_prims(2)


SHELL_CHECK = r"""
#include "topology.hpp"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
using namespace hyb;
int main( int argc, char** argv )
{
   // prints: vertices cells over-shared-faces boundary-faces boundary-off-sphere min-volume total-volume
   const int ntan = atoi( argv[1] ), nrad = atoi( argv[2] );
   const double rmin = 0.55, rmax = 1.0;
   std::vector< std::array< double, 3 > > V;
   std::vector< std::array< int, 4 > >    T;
   meshSphericalShell( ntan, nrad, rmin, rmax, V, T );
   std::map< std::array< int, 3 >, int > fc;
   double vmin = 1e300, vtot = 0;
   for ( auto& t : T )
   {
      double a[3][3];
      for ( int k = 0; k < 3; ++k )
         for ( int d = 0; d < 3; ++d )
            a[k][d] = V[t[k + 1]][d] - V[t[0]][d];
      const double det = a[0][0] * ( a[1][1] * a[2][2] - a[1][2] * a[2][1] ) - a[0][1] * ( a[1][0] * a[2][2] - a[1][2] * a[2][0] ) +
                         a[0][2] * ( a[1][0] * a[2][1] - a[1][1] * a[2][0] );
      vmin = std::min( vmin, std::fabs( det ) / 6 );
      vtot += std::fabs( det ) / 6;
      const int f[4][3] = { { t[0], t[1], t[2] }, { t[0], t[1], t[3] }, { t[0], t[2], t[3] }, { t[1], t[2], t[3] } };
      for ( auto& ff : f )
      {
         std::array< int, 3 > k = { ff[0], ff[1], ff[2] };
         std::sort( k.begin(), k.end() );
         fc[k]++;
      }
   }
   int over = 0, bdry = 0, off = 0;
   for ( auto& kv : fc )
   {
      if ( kv.second > 2 ) ++over;
      if ( kv.second == 1 )
      {
         ++bdry;
         for ( int v : kv.first )
         {
            const double r = std::sqrt( V[v][0] * V[v][0] + V[v][1] * V[v][1] + V[v][2] * V[v][2] );
            if ( std::fabs( r - rmin ) > 1e-12 && std::fabs( r - rmax ) > 1e-12 ) ++off;
         }
      }
   }
   printf( "%zu %zu %d %d %d %.17g %.17g\n", V.size(), T.size(), over, bdry, off, vmin, vtot );
   return 0;
}
"""


@pytest.mark.parametrize("ntan,nrad", [(2, 2), (3, 2), (5, 4)])
def test_spherical_shell_mesh(tmp_path, ntan, nrad):
    """meshSphericalShell: the reference's cell and vertex counts, a conforming
    tetrahedralisation (no face shared by more than two cells), boundary faces only on the
    two spheres, no degenerate cell, and a volume close to the shell's (it grows towards the
    exact one as the sphere is refined)."""
    src = tmp_path / "shell_check.cpp"
    src.write_text(SHELL_CHECK)
    exe = tmp_path / "shell_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(PKG, "csrc"), str(src),
                    os.path.join(PKG, "csrc", "topology.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), str(ntan), str(nrad)], capture_output=True, text=True, check=True).stdout.split()
    nv, nc, over, bdry, off = map(int, out[:5])
    vmin, vtot = map(float, out[5:])
    n = ntan - 1
    assert nc == 60 * n * n * (nrad - 1)
    assert nv == (10 * n * n + 2) * nrad
    assert over == 0 and off == 0
    assert bdry == 2 * 20 * n * n
    assert vmin > 0
    exact = 4.0 / 3.0 * np.pi * (1.0 - 0.55 ** 3)
    assert 0.5 * exact < vtot < exact


GMSH_CHECK = r"""
#include "topology.hpp"
#include <cstdio>
#include <stdexcept>
using namespace hyb;
int main( int argc, char** argv )
{
   std::vector< std::array< double, 3 > > V;
   std::vector< std::array< int, 4 > >    T;
   try
   {
      readGmsh( argv[1], V, T );
   } catch ( const std::exception& e )
   {
      printf( "error %s\n", e.what() );
      return 0;
   }
   printf( "%zu %zu\n", V.size(), T.size() );
   for ( auto& v : V )
      printf( "%.17g %.17g %.17g\n", v[0], v[1], v[2] );
   for ( auto& t : T )
      printf( "%d %d %d %d\n", t[0], t[1], t[2], t[3] );
   return 0;
}
"""


@pytest.fixture(scope="module")
def gmsh_exe(tmp_path_factory):
    d = tmp_path_factory.mktemp("gmsh")
    src = d / "gmsh_check.cpp"
    src.write_text(GMSH_CHECK)
    exe = d / "gmsh_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(PKG, "csrc"), str(src),
                    os.path.join(PKG, "csrc", "topology.cpp"), "-o", str(exe)], check=True)
    return str(exe)


@pytest.mark.parametrize("name", ["tet_1el", "pyramid_4el", "regular_octahedron_8el", "cube_6el"])
def test_gmsh_reader_matches_reference_order(tmp_path, gmsh_exe, write_gmsh, name):
    """readGmsh (MeshInfo::fromGmshFile): vertices in file-id order, tetrahedra in the
    lexicographic order of their vertex lists, whatever the order in the file. The golden
    arrays are the reference's meshes in exactly that order; here the vertices of each
    tetrahedron are permuted in the file, so the check is on the sorted lists."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "reference_meshes.npz"))
    coords, tets = g[name + "_coords"], g[name + "_tets"]
    path = tmp_path / (name + ".msh")
    write_gmsh(path, coords, tets, seed=len(tets), permute_cells=True)
    out = subprocess.run([gmsh_exe, str(path)], capture_output=True, text=True, check=True).stdout.split("\n")
    nv, nt = map(int, out[0].split())
    assert (nv, nt) == (len(coords), len(tets))
    V = np.array([list(map(float, l.split())) for l in out[1:1 + nv]])
    T = np.array([list(map(int, l.split())) for l in out[1 + nv:1 + nv + nt]])
    assert np.array_equal(V, coords)
    want = sorted(tuple(sorted(t)) for t in tets)
    assert sorted(tuple(sorted(t)) for t in T) == want
    assert [tuple(t) for t in T] == sorted(tuple(t) for t in T)


def test_gmsh_reader_rejects_unsupported_files(tmp_path, gmsh_exe):
    """The reference reader accepts only format 2.2 ASCII and element types 1, 2, 4, 15."""
    cases = {
        "v4.msh": "$MeshFormat\n4.1 0 8\n$EndMeshFormat\n",
        "binary.msh": "$MeshFormat\n2.2 1 8\n$EndMeshFormat\n",
        "hex.msh": "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n4\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n"
                   "$EndNodes\n$Elements\n1\n1 5 0 1 2 3 4 1 2 3 4\n$EndElements\n",
        "unknown_node.msh": "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n4\n1 0 0 0\n2 1 0 0\n3 0 1 0\n"
                            "4 0 0 1\n$EndNodes\n$Elements\n1\n1 4 0 1 2 3 9\n$EndElements\n",
    }
    for fname, text in cases.items():
        p = tmp_path / fname
        p.write_text(text)
        out = subprocess.run([gmsh_exe, str(p)], capture_output=True, text=True, check=True).stdout
        assert out.startswith("error"), (fname, out)


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_chebyshev_coefficients(lib, oracle_mod, order):
    """ChebyshevSmoother::setupCoefficients: the product's power-basis coefficients equal the
    oracle's, and 1 - l p(l) is the scaled Chebyshev polynomial T_k((th - l)/de)/T_k(th/de)
    on the eigenvalue interval (host code, no device call)."""
    import hyteg_b200 as H

    rho = 1.7
    lo, hi = 0.3 * rho, 1.2 * rho
    w = H.chebyshev_coefficients(order, lo, hi)
    np.testing.assert_allclose(w, oracle_mod.chebyshev_coefficients(order, lo, hi), rtol=1e-14)
    th, de = (hi + lo) / 2, (hi - lo) / 2
    lam = np.linspace(0.0, hi, 11)
    r = 1 - lam * np.polyval(w[::-1], lam)
    Tk = np.polynomial.chebyshev.Chebyshev.basis(order)
    np.testing.assert_allclose(r, Tk((th - lam) / de) / Tk(th / de), atol=1e-12)
    with pytest.raises(H.HybError):
        H.chebyshev_coefficients(6, lo, hi)
