"""Blending (curved shell) operator of the oracle, pinned to the reference:
IcosahedralShellMap (evalF, evalDF, vertex classification incl. skew cells) and the
p1_div_k_grad_blending_q3 element matrix must equal the reference's own code compiled from
its tree (golden fixture tests/golden/blend_shell_ntan3_nrad2.npz, made by
tests/golden/make_blend_golden.py); the assembled operator must annihilate constants,
be symmetric, and let the multigrid solver converge."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "blend_shell_ntan3_nrad2.npz")


@pytest.fixture(scope="module")
def shell(oracle_mod):
    g = np.load(GOLD)
    return oracle_mod, g, oracle_mod.Oracle(g["V"], g["T"], 2)


def test_shell_map_matches_reference(shell):
    O, g, orc = shell
    for c in range(len(g["T"])):
        F, DF = orc.shell_map(c, g["x"][c])
        np.testing.assert_allclose(F, g["F"][c], rtol=0, atol=1e-14 * np.abs(g["F"][c]).max())
        np.testing.assert_allclose(DF.reshape(9), g["DF"][c], rtol=0, atol=1e-14 * np.abs(g["DF"][c]).max())


def test_blend_element_matrix_matches_reference(shell):
    O, g, orc = shell
    for c in range(len(g["T"])):
        for a, alpha in enumerate(g["alphas"]):
            A = orc.blend_element_matrix(c, g["X"][c], alpha)
            ref = g["A"][c, a].reshape(4, 4)
            np.testing.assert_allclose(A, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_blend_matches_compiled_reference_when_present(shell):
    """Direct comparison with oracle/_ref (only where the reference tree was compiled)."""
    import ctypes

    O, g, orc = shell
    path = os.path.join(O.HERE, "_ref", "libhyteg_refblend.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref/libhyteg_refblend.so not built here")
    R = ctypes.CDLL(path)
    P, I, D, LG = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long
    R.ref_blend_element_matrix.argtypes = [P, LG, P, LG, I, P, D, P]
    V, T = np.ascontiguousarray(g["V"]), np.ascontiguousarray(g["T"])
    rng = np.random.default_rng(7)
    for c in rng.choice(len(T), 40, replace=False):
        # a well-shaped random sub-tet of the cell (not a lattice micro-tet)
        X = np.ascontiguousarray((0.6 * np.eye(4) + 0.4 * rng.dirichlet([1, 1, 1, 1], 4)) @ V[T[c]])
        ref = np.zeros(16)
        assert R.ref_blend_element_matrix(V.ctypes.data, len(V), T.ctypes.data, len(T), int(c), X.ctypes.data, 2.0,
                                          ref.ctypes.data) == 0
        np.testing.assert_allclose(orc.blend_element_matrix(int(c), X, 2.0).reshape(16), ref, rtol=0,
                                   atol=1e-12 * np.abs(ref).max())


def test_non_shell_mesh_is_rejected(oracle_mod):
    O = oracle_mod
    coords, tets = O.mesh_cuboid(1, 1, 1)
    orc = O.Oracle(coords, tets, 1)
    with pytest.raises(ValueError):
        orc.op_blend_div_k_grad(0.0)


def test_blend_operator_annihilates_constants_and_is_symmetric(shell):
    O, g, orc = shell
    op = orc.op_blend_div_k_grad(5.0)
    L = 2
    n = orc.n(L)
    Au = orc.apply(np.ones(n), L, flag=O.ALL, op=op)
    assert np.abs(Au).max() < 1e-12 * np.abs(orc.apply(np.linspace(0, 1, n), L, flag=O.ALL, op=op)).max()
    rng = np.random.default_rng(3)
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    lhs = y @ orc.apply(x, L, flag=O.ALL, op=op)
    rhs = x @ orc.apply(y, L, flag=O.ALL, op=op)
    assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + abs(rhs))


def test_blend_gmg_converges(shell):
    O, g, orc = shell
    op = orc.op_blend_div_k_grad(5.0)
    L = 2
    _, bc = orc.info(L)
    rng = np.random.default_rng(11)
    b = rng.uniform(-1, 1, orc.n(L)) * (bc == O.INNER)
    x = np.zeros(orc.n(L))
    r0 = np.linalg.norm(b)
    orc.gmg(x, b, 0, L, max_cycles=6, op=op)
    r = b - orc.apply(x, L, op=op)
    r[bc != O.INNER] = 0
    assert np.linalg.norm(r) < 1e-3 * r0
