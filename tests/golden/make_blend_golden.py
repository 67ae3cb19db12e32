"""Generates tests/golden/blend_shell_ntan3_nrad2.npz: outputs of the reference's own
IcosahedralShellMap (evalF, evalDF) and p1_div_k_grad_blending_q3 form (integrateAll),
compiled unchanged from the reference tree by `make -C oracle ref` into
oracle/_ref/libhyteg_refblend.so, on the spherical shell ntan = 3, nrad = 2, radii
0.55-1.0 (240 macro-tets, meshSphericalShell of hyteg-vara_b200/csrc/topology.cpp).

Per cell: the map at one seeded interior point, and the element matrix of one level-2
micro-tet for k = 1 (alpha = 0) and k = exp(5 (1 - |x|)) (alpha = 5).

    HYTEG_REFERENCE_ROOT=<reference checkout> make -C oracle ref && python tests/golden/make_blend_golden.py
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CSRC = os.path.join(ROOT, "hyteg-vara_b200", "csrc")
OUT = os.path.join(HERE, "blend_shell_ntan3_nrad2.npz")

MESH_MAIN = r"""
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


def shell_mesh(ntan, nrad, rmin, rmax):
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "m.cpp"), os.path.join(d, "m")
        open(src, "w").write(MESH_MAIN)
        subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, src, os.path.join(CSRC, "topology.cpp"), "-o", exe],
                       check=True)
        lines = subprocess.run([exe, str(ntan), str(nrad), repr(rmin), repr(rmax)], check=True, capture_output=True,
                               text=True).stdout.split("\n")
    nv, nt = map(int, lines[0].split())
    V = np.array([[float(x) for x in l.split()] for l in lines[1:1 + nv]])
    T = np.array([[int(x) for x in l.split()] for l in lines[1 + nv:1 + nv + nt]], dtype=np.int64)
    return V, T


def main():
    R = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libhyteg_refblend.so"))
    P, I, D, LG = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long
    R.ref_shell_map_eval.argtypes = [P, LG, P, LG, I, P, P, P]
    R.ref_blend_element_matrix.argtypes = [P, LG, P, LG, I, P, D, P]
    p = lambda a: a.ctypes.data_as(P)  # noqa: E731
    V, T = shell_mesh(3, 2, 0.55, 1.0)
    rng = np.random.default_rng(2024)
    nt = len(T)
    x = np.zeros((nt, 3))
    F = np.zeros((nt, 3))
    DF = np.zeros((nt, 9))
    X = np.zeros((nt, 4, 3))
    alphas = np.array([0.0, 5.0])
    A = np.zeros((nt, len(alphas), 16))
    # the level-2 micro-tets of a cell: vertex v0 + (v_k - v0) * i_k / 4 at integer offsets
    shapes = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]],
                       [[1, 0, 0], [1, 1, 0], [0, 1, 0], [1, 0, 1]],
                       [[2, 1, 0], [1, 1, 1], [1, 2, 0], [1, 1, 0]]])
    for c in range(nt):
        cv = V[T[c]]
        x[c] = rng.dirichlet([1, 1, 1, 1]) @ cv
        assert R.ref_shell_map_eval(p(V), len(V), p(T), nt, c, p(x[c]), p(F[c]), p(DF[c])) == 0
        sh = shapes[c % len(shapes)]
        for j in range(4):
            X[c, j] = cv[0] + (cv[1] - cv[0]) / 4 * sh[j][0] + (cv[2] - cv[0]) / 4 * sh[j][1] + \
                (cv[3] - cv[0]) / 4 * sh[j][2]
        for a, alpha in enumerate(alphas):
            Xc = np.ascontiguousarray(X[c])
            assert R.ref_blend_element_matrix(p(V), len(V), p(T), nt, c, p(Xc), alpha, p(A[c, a])) == 0
    np.savez_compressed(OUT, V=V, T=T, x=x, F=F, DF=DF, X=X, alphas=alphas, A=A)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
