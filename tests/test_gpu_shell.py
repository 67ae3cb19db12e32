"""Spherical-shell meshes on the GPU against the CPU oracle: the shell storage's mesh is
handed to the oracle, and the constant-coefficient apply, the device-evaluated shell
coefficient (radial profile times lognormal noise) and a V(2,2) cycle must agree (1e-12
for applies, 1e-10 for the cycle, the tolerances of the other parity tests)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shell(oracle_mod):
    import hyteg_b200 as H

    H.load()
    L = 3
    st = H.PrimitiveStorage.spherical_shell(3, 2, 0.55, 1.0, L)
    coords, tets = st.mesh()
    orc = oracle_mod.Oracle(coords, tets, L)
    return H, st, orc, L


def close(a, b, rtol):
    err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    assert err <= rtol, f"max relative error {err:.3e} > {rtol:.1e}"


def test_shell_counts_and_boundary(shell):
    H, st, orc, L = shell
    nv, ne, nf, nc = st.counts()
    assert nc == 60 * 4 * 1 and nv == (10 * 4 + 2) * 2
    for l in range(L + 1):
        assert st.num_dofs(l) == orc.n(l)
    # every vertex lies on one of the two spheres
    coords, _ = st.mesh()
    r = np.sqrt((coords ** 2).sum(axis=1))
    assert np.all(np.isclose(r, 0.55) | np.isclose(r, 1.0))


def test_shell_laplace_apply_matches_oracle(shell):
    H, st, orc, L = shell
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    rng = np.random.default_rng(4)
    for level in range(L + 1):
        x = rng.uniform(-1, 1, orc.n(level))
        fs, fd = H.P1Function("s", st, 0, L), H.P1Function("d", st, 0, L)
        fs.set(x, level)
        A.apply(fs, fd, level, H.ALL)
        close(fd.get(level), orc.apply(x, level, flag=H.ALL), 1e-12)


def test_shell_coefficient_apply_and_vcycle_match_oracle(shell):
    import hyb_inputs as I

    H, st, orc, L = shell
    w, ph = I.grf_features(0.2, 2, 64)
    A = H.P1ElementwiseDivKGradOperator.random_features(st, 0, L, w, ph, 0.5, radial=5.0)
    kv = [I.shell_coefficient(orc.coords_of(l)) for l in range(L + 1)]
    op = orc.op_divkgrad(kv)
    rng = np.random.default_rng(6)
    for level in range(L + 1):
        x = rng.uniform(-1, 1, orc.n(level))
        fs, fd = H.P1Function("s", st, 0, L), H.P1Function("d", st, 0, L)
        fs.set(x, level)
        A.apply(fs, fd, level, H.ALL)
        close(fd.get(level), orc.apply(x, level, flag=H.ALL, op=op), 1e-12)
    m, labels = st.colouring()
    b = rng.uniform(-1, 1, orc.n(L))
    fx, fb = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
    fb.set(b, L)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 2, 2, 1.0)
    gmg.solve(fx, fb, L)
    x = np.zeros(orc.n(L))
    orc.gmg(x, b, 0, L, pre=2, post=2, relax=1.0, smoother=1, labels=labels, m=m, coarse_tol=1e-12, max_cycles=1, op=op)
    close(fx.get(L), x, 1e-10)


def test_config5_mesh_apply_and_vcycle_match_oracle(oracle_mod):
    """The benchmarked shell shape (ntan 5, radii 0.55 to 1.0 in 3 radial layers, 2880
    macro-tets) at level 4, radial coefficient exp(5 (1 - r)) times lognormal noise: the
    coefficient apply and one V(2,2) cycle against the oracle."""
    import hyb_inputs as I
    import hyteg_b200 as H

    H.load()
    L = 4
    st = H.PrimitiveStorage.spherical_shell(5, 4, 0.55, 1.0, L)
    coords, tets = st.mesh()
    assert len(tets) == 2880
    orc = oracle_mod.Oracle(coords, tets, L)
    w, ph = I.grf_features(0.2, 2, 64)
    A = H.P1ElementwiseDivKGradOperator.random_features(st, 0, L, w, ph, 0.5, radial=5.0)
    op = orc.op_divkgrad([I.shell_coefficient(orc.coords_of(l)) for l in range(L + 1)])
    rng = np.random.default_rng(9)
    x = rng.uniform(-1, 1, orc.n(L))
    fs, fd = H.P1Function("s", st, 0, L), H.P1Function("d", st, 0, L)
    fs.set(x, L)
    A.apply(fs, fd, L, H.ALL)
    close(fd.get(L), orc.apply(x, L, flag=H.ALL, op=op), 1e-12)
    m, labels = st.colouring()
    b = rng.uniform(-1, 1, orc.n(L))
    fx, fb = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
    fb.set(b, L)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 2, 2, 1.0)
    gmg.solve(fx, fb, L)
    xo = np.zeros(orc.n(L))
    orc.gmg(xo, b, 0, L, pre=2, post=2, relax=1.0, smoother=1, labels=labels, m=m, coarse_tol=1e-12, max_cycles=1,
            op=op)
    close(fx.get(L), xo, 1e-10)
