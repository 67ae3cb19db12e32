"""Generates tests/golden/shell_mesh_reference.npz: spherical-shell meshes of the reference's
own MeshInfo::meshSphericalShell (src/hyteg/mesh/MeshGenSphericalShell.cpp, SHELLMESH_CLASSIC),
compiled unchanged from the reference tree by `make -C oracle ref` into
oracle/_ref/libhyteg_refmesh.so: vertex coordinates in vertex-id order and cells in the order
of the reference's cell map, for (ntan, nrad) = (3, 2), (5, 3), (5, 4), radii 0.55 .. 1.0.

    HYTEG_REFERENCE_ROOT=<reference checkout> make -C oracle ref && python tests/golden/make_shell_mesh_golden.py
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "shell_mesh_reference.npz")
CASES = [(3, 2), (5, 3), (5, 4)]


def main():
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libhyteg_refmesh.so"))
    f = lib.ref_mesh_spherical_shell
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    out = {}
    for ntan, nrad in CASES:
        n = np.zeros(2, np.int64)
        assert f(ntan, nrad, 0.55, 1.0, n.ctypes.data, None, None) == 0
        coords = np.zeros((n[0], 3))
        tets = np.zeros((n[1], 4), np.int64)
        assert f(ntan, nrad, 0.55, 1.0, n.ctypes.data, coords.ctypes.data, tets.ctypes.data) == 0
        out[f"ntan{ntan}_nrad{nrad}_coords"] = coords
        out[f"ntan{ntan}_nrad{nrad}_tets"] = tets
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
