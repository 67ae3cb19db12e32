"""Generates tests/golden/divkgrad_affine_q3.npz: element matrices of the reference's own
p1_div_k_grad_affine_q3 form (integrateAll, tetrahedron; the 5-point degree-3 rule "Yu 2"),
compiled unchanged from the reference tree by `make -C oracle ref` into
oracle/_ref/libhyteg_refblend.so, on seeded random tetrahedra with two coefficient callbacks:

  kind 0: the P1 interpolant of random positive nodal values k4 on the tetrahedron (what the
          variable-coefficient operator's nodal coefficient means);
  kind 1: k(x) = tanh(2 (x - 1/2)) + 2, the coefficient of the reference's
          tests/hyteg/convergence/ElementwiseDivKGradCGConvergenceTest.cpp.

    HYTEG_REFERENCE_ROOT=<reference checkout> make -C oracle ref && python tests/golden/make_divkgrad_golden.py
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "divkgrad_affine_q3.npz")


def main():
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libhyteg_refblend.so"))
    f = lib.ref_divkgrad_affine_element_matrix
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    rng = np.random.default_rng(7)
    X, K4, A0, A1 = [], [], [], []
    while len(X) < 24:
        x = rng.uniform(-1.0, 1.0, size=(4, 3))
        vol = abs(np.linalg.det(x[1:] - x[0])) / 6.0
        if vol < 0.02:
            continue  # keep the tetrahedra well shaped
        k4 = rng.uniform(0.1, 3.0, size=4)
        out = []
        for kind in (0, 1):
            a = np.zeros(16)
            assert f(np.ascontiguousarray(x).ctypes.data, kind, np.ascontiguousarray(k4).ctypes.data,
                     a.ctypes.data) == 0
            out.append(a.reshape(4, 4))
        X.append(x)
        K4.append(k4)
        A0.append(out[0])
        A1.append(out[1])
    np.savez(OUT, X=np.array(X), k4=np.array(K4), A_interp=np.array(A0), A_tanh=np.array(A1))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
