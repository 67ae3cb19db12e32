"""Pin the CPU oracle to the reference: its results must equal the reference's own
generated kernels and FEniCS form on the committed golden fixtures
(tests/golden/make_golden.py), plus the reference tests' known answers."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def tet_size(w):
    return (w + 2) * (w + 1) * w // 6


def cell_idx(width, x, y, z):
    wms = width - z
    return tet_size(width) - tet_size(wms) + y * (wms + 1) - ((y + 1) * y) // 2 + x


def interior_points(N):
    for z in range(1, N + 1):
        for y in range(1, N - z + 1):
            for x in range(1, N - y - z):
                yield x, y, z


def test_stencils_match_reference_fenics_assembly(oracle_mod):
    O = oracle_mod
    g = np.load(os.path.join(GOLD, "stencils_cube1.npz"))
    o = O.Oracle(g["coords"], g["tets"], int(g["levels"].max()))
    for li, L in enumerate(g["levels"]):
        for c in range(len(g["tets"])):
            ref = g["stencils"][li, c]
            np.testing.assert_allclose(o.cell_stencil(int(L), c, 0), ref, rtol=0, atol=1e-13 * np.abs(ref).max())


def test_cell_apply_matches_generated_kernel(oracle_mod):
    O = oracle_mod
    g = np.load(os.path.join(GOLD, "cell_kernels_L4.npz"))
    s = np.load(os.path.join(GOLD, "stencils_cube1.npz"))
    L = int(g["level"])
    N = 1 << L
    o = O.Oracle(s["coords"], s["tets"], L)
    cm = o.closure_map(L, 0)
    x = np.zeros(o.n(L))
    x[cm] = g["src"]
    for add, key in ((False, "apply_replace"), (True, "apply_add")):
        y = np.zeros(o.n(L))
        y[cm] = g["dst0"]
        o.apply(x, L, flag=O.ALL, dst=y, add=add)
        for (px, py, pz) in interior_points(N):
            i = cell_idx(N + 1, px, py, pz)
            assert abs(y[cm[i]] - g[key][i]) <= 1e-13 * (1 + abs(g[key][i]))


@pytest.mark.parametrize("backwards", [False, True])
@pytest.mark.parametrize("relax", [1.0, 0.8])
def test_cell_sor_matches_generated_kernel(oracle_mod, relax, backwards):
    """Single macro-tet: every face/edge/vertex is Dirichlet, so the reference-order SOR
    reduces to the generated lexicographic cell sweep (sor_3D_macrocell_P1.cpp, and
    sor_3D_macrocell_P1_backwards.cpp for the backward sweep)."""
    O = oracle_mod
    g = np.load(os.path.join(GOLD, "cell_kernels_L4.npz"))
    s = np.load(os.path.join(GOLD, "stencils_cube1.npz"))
    L = int(g["level"])
    N = 1 << L
    t0 = s["tets"][0]
    o = O.Oracle(s["coords"][t0], np.array([[0, 1, 2, 3]]), L)
    cm = o.closure_map(L, 0)
    x = np.zeros(o.n(L))
    b = np.zeros(o.n(L))
    x[cm] = g["src"]
    b[cm] = g["rhs"]
    o.sor_ref(x, b, L, relax=relax, flag=O.INNER, backwards=backwards)
    ref = g[f"sor_relax{relax}_bw{int(backwards)}"]
    got = x[cm]
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-13)


def test_transfers_match_generated_kernels(oracle_mod):
    """Per-cell push/pull kernels with 1/#neighbour-cell scaling, summed over cells
    (communicateAdditively), equal the oracle's global prolongation/restriction."""
    O = oracle_mod
    g = np.load(os.path.join(GOLD, "transfer_cube1_L3.npz"))
    s = np.load(os.path.join(GOLD, "stencils_cube1.npz"))
    cl = int(g["coarse_level"])
    o = O.Oracle(s["coords"], s["tets"], cl + 1)
    fine_sum = np.zeros(o.n(cl + 1))
    coarse_sum = np.zeros(o.n(cl))
    for c in range(len(s["tets"])):
        np.add.at(fine_sum, o.closure_map(cl + 1, c), g["prolongated"][c])
        np.add.at(coarse_sum, o.closure_map(cl, c), g["restricted"][c])
    pro = o.prolongate(g["coarse"], cl, flag=O.ALL)
    res = o.restrict(g["fine"], cl + 1, flag=O.ALL)
    np.testing.assert_allclose(pro, fine_sum, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(res, coarse_sum, rtol=1e-12, atol=1e-13)


def test_element_stiffness_matches_fenics_form(oracle_mod):
    """The oracle's Laplace stencils are built from its own P1 stiffness; checking the
    single-element stencil of a one-tet mesh at level 0 against tabulate_tensor."""
    O = oracle_mod
    g = np.load(os.path.join(GOLD, "fenics_p1_tet_diffusion.npz"))
    for X, K in zip(g["coords"], g["K"]):
        V = X.reshape(4, 3)
        if abs(np.linalg.det(V[1:] - V[0])) < 1e-3:
            continue
        o = O.Oracle(V, np.array([[0, 1, 2, 3]]), 0)
        K = K.reshape(4, 4)
        for v in range(4):
            e = np.zeros(4)
            e[v] = 1.0
            y = o.apply(e, 0, flag=O.ALL)
            np.testing.assert_allclose(y, K[:, v], rtol=1e-12, atol=1e-13 * np.abs(K).max())


# ---------------------------------------------------------------------------
# Known answers from the reference's own tests
# ---------------------------------------------------------------------------
def test_laplace_of_constant_and_linear_vanishes(oracle_mod):
    """tests/hyteg/P1/P1LaplaceOperator3DTest.cpp:47-134 (discrete L2 < 2.8e-13)."""
    O = oracle_mod
    c, t = O.mesh_cuboid(2, 1, 1)
    for L in (2, 3):
        o = O.Oracle(c, t, L)
        xyz = o.coords_of(L)
        kind, bc = o.info(L)
        for f in (np.ones(len(xyz)), 1 + xyz[:, 0] - 2 * xyz[:, 1] + 3 * xyz[:, 2]):
            y = o.apply(f, L, flag=O.INNER)
            err = np.sqrt(np.sum(y[bc == O.INNER] ** 2) / max(1, np.sum(bc == O.INNER)))
            assert err < 2.8e-13


def test_prolongation_exact_on_linears(oracle_mod):
    """tests/hyteg/vertexdofspace/VertexDoFLinearProlongation3DTest.cpp:48-192 (< 1e-15)."""
    O = oracle_mod
    c, t = O.mesh_cuboid(1, 1, 2)
    o = O.Oracle(c, t, 3)
    f = lambda p: 0.5 + p[:, 0] + 2 * p[:, 1] - p[:, 2]
    for L in (0, 1, 2):
        fine = o.prolongate(f(o.coords_of(L)), L, flag=O.ALL)
        assert np.abs(fine - f(o.coords_of(L + 1))).max() < 1e-14
        # prolongateAndAdd == prolongate + add
        base = np.random.default_rng(L).uniform(size=o.n(L + 1))
        added = o.prolongate(f(o.coords_of(L)), L, fine=base.copy(), flag=O.ALL, add=True)
        assert np.abs(added - (base + fine)).max() < 1e-15 * 8


def test_restriction_is_transpose_of_prolongation(oracle_mod):
    O = oracle_mod
    c, t = O.mesh_cuboid(2, 2, 1)
    o = O.Oracle(c, t, 3)
    rng = np.random.default_rng(3)
    r, e = rng.uniform(size=o.n(3)), rng.uniform(size=o.n(2))
    lhs = r @ o.prolongate(e, 2, flag=O.ALL)
    rhs = e @ o.restrict(r, 3, flag=O.ALL)
    assert abs(lhs - rhs) <= 1e-13 * abs(lhs)


def test_gmg_convergence_rate_reference_order_sor(oracle_mod):
    """tests/hyteg/convergence/P1GMG3DConvergenceTest.cpp:30-150 on its own mesh
    (regular_octahedron_8el), levels 0..3: u random inside, exact Dirichlet values
    sin(x) sinh(y) z, f = 0, V(3,3) with Gauss-Seidel, CG coarse solve; every cycle must
    cut the squared discrete L2 residual by more than 1/3.2e-2."""
    O = oracle_mod
    g = np.load(os.path.join(GOLD, "reference_meshes.npz"))
    o = O.Oracle(g["regular_octahedron_8el_coords"], g["regular_octahedron_8el_tets"], 3)
    xyz = o.coords_of(3)
    kind, bc = o.info(3)
    x = np.random.default_rng(0).uniform(0, 1, o.n(3))
    exact = np.sin(xyz[:, 0]) * np.sinh(xyz[:, 1]) * xyz[:, 2]
    x[bc == O.DIRICHLET] = exact[bc == O.DIRICHLET]
    b = np.zeros(o.n(3))
    _, hist = o.gmg(x, b, 0, 3, pre=3, post=3, relax=1.0, smoother=0, max_cycles=4)
    ratios = (hist[1:] / hist[:-1]) ** 2
    assert np.all(ratios < 3.2e-2), ratios


def test_symmetric_multicolour_sor_is_a_symmetric_operator(oracle_mod):
    """A forward multicolour sweep followed by the backward one (the passes in reverse
    order) from a zero start is b -> M^-1 b with M symmetric (symmetric SOR), because the
    stiffness matrix is symmetric: <S b1, b2> == <b1, S b2> over the inner DoFs."""
    O = oracle_mod
    c, t = O.mesh_cuboid(2, 1, 1, hi=(2.0, 1.0, 1.0))
    L = 3
    o = O.Oracle(c, t, L)
    kind, bc = o.info(L)
    inner = bc == O.INNER
    labels, m = np.arange(len(c)), len(c)  # distinct vertex labels: a valid multicolouring
    rng = np.random.default_rng(5)
    for relax in (1.0, 1.3):
        S = []
        bs = []
        for _ in range(2):
            b = rng.uniform(-1, 1, o.n(L)) * inner
            x = np.zeros(o.n(L))
            o.sor_colored(x, b, L, labels, m, relax=relax)
            o.sor_colored(x, b, L, labels, m, relax=relax, backwards=True)
            S.append(x)
            bs.append(b)
        lhs, rhs = S[0] @ bs[1], bs[0] @ S[1]
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (relax, lhs, rhs)
        # the forward sweep alone is not symmetric
        x0, x1 = np.zeros(o.n(L)), np.zeros(o.n(L))
        o.sor_colored(x0, bs[0], L, labels, m, relax=relax)
        o.sor_colored(x1, bs[1], L, labels, m, relax=relax)
        assert abs(x0 @ bs[1] - bs[0] @ x1) > 1e-8 * abs(x0 @ bs[1])


@pytest.mark.parametrize("smoother", [3, 4])
@pytest.mark.parametrize("cycle", ["V", "W"])
def test_gmg_convergence_symmetric_sor_and_w_cycles(oracle_mod, smoother, cycle):
    """P1GMG3DConvergenceTest.cpp's setting (regular_octahedron_8el, levels 0..3, V(3,3)) with
    SymmetricSORSmoother, as V- and W-cycles: every cycle must beat the reference test's
    bound 3.2e-2 on the squared residual ratio, and the W-cycle must not converge slower
    than the V-cycle."""
    O = oracle_mod
    g = np.load(os.path.join(GOLD, "reference_meshes.npz"))
    c, t = g["regular_octahedron_8el_coords"], g["regular_octahedron_8el_tets"]
    o = O.Oracle(c, t, 3)
    labels, m = np.arange(len(c)), len(c)  # distinct vertex labels: a valid multicolouring
    xyz = o.coords_of(3)
    kind, bc = o.info(3)
    x0 = np.random.default_rng(0).uniform(0, 1, o.n(3))
    exact = np.sin(xyz[:, 0]) * np.sinh(xyz[:, 1]) * xyz[:, 2]
    x0[bc == O.DIRICHLET] = exact[bc == O.DIRICHLET]
    b = np.zeros(o.n(3))
    rates = {}
    for cyc in ("V", cycle):
        _, hist = o.gmg(x0.copy(), b, 0, 3, pre=3, post=3, relax=1.0, smoother=smoother, labels=labels, m=m,
                        max_cycles=4, cycle=cyc)
        rates[cyc] = (hist[1:] / hist[:-1]) ** 2
        assert np.all(rates[cyc] < 3.2e-2), (cyc, rates[cyc])
    assert rates[cycle].max() <= rates["V"].max() * (1 + 1e-9)


@pytest.mark.parametrize("order", [2, 3, 4])
def test_gmg_convergence_chebyshev(oracle_mod, order):
    """ChebyshevSmoother in the P1GMG3DConvergenceTest.cpp setting (regular_octahedron_8el,
    levels 0..3, V(3,3)): coefficients from the power-iteration estimate of D^-1 A's spectral
    radius (chebyshev::estimateRadius, [0.3 rho, 1.2 rho]); the estimate lies in the
    interval's admissible range, and every cycle reduces the residual."""
    O = oracle_mod
    g = np.load(os.path.join(GOLD, "reference_meshes.npz"))
    o = O.Oracle(g["regular_octahedron_8el_coords"], g["regular_octahedron_8el_tets"], 3)
    rho = o.spectral_radius(3, 40, np.random.default_rng(1).uniform(0, 1, o.n(3)))
    assert 1.0 < rho < 2.5  # D^-1 A of the P1 Laplacian: spectrum in (0, 2] plus boundary rows
    o.set_chebyshev(order, 0.3 * rho, 1.2 * rho)
    xyz = o.coords_of(3)
    kind, bc = o.info(3)
    x = np.random.default_rng(0).uniform(0, 1, o.n(3))
    exact = np.sin(xyz[:, 0]) * np.sinh(xyz[:, 1]) * xyz[:, 2]
    x[bc == O.DIRICHLET] = exact[bc == O.DIRICHLET]
    _, hist = o.gmg(x, np.zeros(o.n(3)), 0, 3, pre=3, post=3, smoother=5, max_cycles=4)
    ratios = hist[1:] / hist[:-1]
    assert np.all(ratios < 0.1), ratios
