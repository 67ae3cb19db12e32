"""The variable-coefficient operator with the coefficient integrated as the reference's form
does it (p1_div_k_grad_affine_q3: the callback at the 5 quadrature points of every micro-tet,
on every level) against the oracle's callback operator, whose form is pinned to the
compiled reference form: apply 1e-12, multicolour SOR 1e-11, a V(3,3) cycle 1e-10 (the
tolerances of the other parity tests), FP32 rows 1e-5; and the reference's
ElementwiseDivKGradCGConvergenceTest (P1, 3D) with its own coefficient semantics."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def close(a, b, rtol):
    err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    assert err <= rtol, f"max relative error {err:.3e} > {rtol:.1e}"


@pytest.fixture(scope="module")
def cube(oracle_mod):
    import hyb_inputs as I
    import hyteg_b200 as H

    H.load()
    L = 4
    coords, tets = oracle_mod.mesh_cuboid(2, 1, 1, hi=(2.0, 1.0, 1.0))
    st = H.PrimitiveStorage(coords, tets, L)
    orc = oracle_mod.Oracle(coords, tets, L)
    w, ph = I.grf_features(0.2, 1, 64)
    return H, st, orc, L, w, ph


@pytest.mark.parametrize("kind", [1, 2])
def test_quadrature_apply_and_sor_match_oracle(cube, kind):
    H, st, orc, L, w, ph = cube
    A = H.P1ElementwiseDivKGradOperator.quadrature(st, 0, L, kind, w, ph, sigma=1.0, radial=0.5)
    op = orc.op_divkgrad_callback(kind, w, ph, sigma=1.0, radial=0.5)
    m, labels = st.colouring()
    rng = np.random.default_rng(31 + kind)
    for level in range(L + 1):
        x, b = rng.uniform(-1, 1, orc.n(level)), rng.uniform(-1, 1, orc.n(level))
        fs, fd, fb = (H.P1Function(n, st, 0, L) for n in "sdb")
        fs.set(x, level)
        fb.set(b, level)
        A.apply(fs, fd, level, H.ALL)
        close(fd.get(level), orc.apply(x, level, flag=H.ALL, op=op), 1e-12)
        A.residual(fs, fb, fd, level, H.INNER | H.NEUMANN)
        r = b - orc.apply(x, level, flag=H.INNER | H.NEUMANN, op=op)
        mask = (orc.info(level)[1] & (H.INNER | H.NEUMANN)) != 0
        if mask.any():  # level 0 of this mesh has boundary DoFs only
            close(fd.get(level)[mask], r[mask], 1e-12)
        if level >= 1:
            A.smooth_sor(fs, fb, 1.0, level, H.INNER | H.NEUMANN)
            xr = orc.sor_colored(x.copy(), b, level, labels, m, flag=H.INNER | H.NEUMANN, op=op)
            close(fs.get(level), xr, 1e-11)
    # FP32 rows (the mixed solver's single-precision cycles)
    x = rng.uniform(-1, 1, orc.n(L))
    f32s, f32d = H.P1Function("s32", st, 0, L, H.F32), H.P1Function("d32", st, 0, L, H.F32)
    f32s.set(x.astype(np.float32), L)
    A.apply(f32s, f32d, L, H.ALL)
    close(f32d.get(L).astype(np.float64), orc.apply(x, L, flag=H.ALL, op=op), 1e-5)


def test_quadrature_vcycle_and_mixed_solve_match_oracle(cube):
    """One V(3,3) cycle equals the oracle's multicolour cycle with the callback operator on
    every level (1e-10); the mixed-precision solve to 1e-8 agrees with the oracle's FP64
    solution (1e-6) in a cycle count within one of the oracle's."""
    H, st, orc, L, w, ph = cube
    import hyb_inputs as I

    A = H.P1ElementwiseDivKGradOperator.quadrature(st, 0, L, 2, w, ph, sigma=1.0)
    op = orc.op_divkgrad_callback(2, w, ph, sigma=1.0)
    m, labels = st.colouring()
    b = I.uniform_rhs(orc.coords_of(L), 3, 2 << L)
    fx, fb = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
    fb.set(b, L)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0)
    gmg.solve(fx, fb, L)
    x = np.zeros(orc.n(L))
    orc.gmg(x, b, 0, L, pre=3, post=3, relax=1.0, smoother=1, labels=labels, m=m, coarse_tol=1e-12, max_cycles=1, op=op)
    close(fx.get(L), x, 1e-10)
    fx.interpolate(0.0, L, flag=H.ALL)
    hist = gmg.solve_to_tolerance(fx, fb, L, 1e-8, max_cycles=60, precision=32)
    assert hist[-1] <= 1e-8
    x_oc = np.zeros(orc.n(L))
    _, h_oc = orc.gmg(x_oc, b, 0, L, pre=3, post=3, smoother=1, labels=labels, m=m, max_cycles=60, rel_tol=1e-8, op=op)
    assert abs((len(hist) - 1) - (len(h_oc) - 1)) <= 1, (hist, h_oc)
    xr = np.zeros(orc.n(L))
    orc.gmg(xr, b, 0, L, pre=3, post=3, smoother=0, max_cycles=100, rel_tol=1e-13, op=op)
    close(fx.get(L), xr, 1e-6)


@pytest.mark.parametrize("level,target", [(3, 1.1e-3), (4, 3.5e-4), (5, 1.0e-4)])
def test_reference_cg_convergence_with_reference_coefficient_semantics(oracle_mod, level, target):
    """ElementwiseDivKGradCGConvergenceTest (tests/hyteg/convergence/
    ElementwiseDivKGradCGConvergenceTest.cpp:41-137), P1, 3D, on tet_1el: -div(k grad u) = f,
    u = sin(2 pi x) sinh(pi y), k = tanh(2 (x - 1/2)) + 2 evaluated at the form's quadrature
    points as the reference does, f = M r, CG to 1e-12; the reference's thresholds on the
    discrete L2 error, and the GPU solution equals the oracle's callback-operator CG
    solution to 1e-9."""
    import hyteg_b200 as H

    O = oracle_mod
    H.load()
    g = np.load(os.path.join(GOLD, "reference_meshes.npz"))
    coords, tets = g["tet_1el_coords"], g["tet_1el_tets"]
    st = H.PrimitiveStorage(coords, tets, level)
    orc = O.Oracle(coords, tets, level)
    alpha, phi = 2.0, 2.0
    xyz = orc.coords_of(level)
    x, y = xyz[:, 0], xyz[:, 1]
    exact = np.sin(phi * np.pi * x) * np.sinh(np.pi * y)
    t0 = np.tanh(alpha * (x - 0.5))
    t1 = phi * alpha * (t0 * t0 - 1.0) * np.cos(phi * np.pi * x)
    t2 = (phi * phi - 1.0) * np.pi * (t0 + 2.0) * np.sin(phi * np.pi * x)
    r = np.pi * (t1 + t2) * np.sinh(np.pi * y)
    f = orc.apply(r, level, flag=O.ALL, op=orc.op_mass())
    _, bc = orc.info(level)
    u0 = np.where((bc & O.DIRICHLET) != 0, exact, 0.0)
    A = H.P1ElementwiseDivKGradOperator.quadrature(st, level, level, 1)
    fu, ff = H.P1Function("u", st, level, level), H.P1Function("f", st, level, level)
    fu.set(u0, level)
    ff.set(f, level)
    it, conv = H.CGSolver(tolerance=1e-12, max_iter=1000).solve(A, fu, ff, level)
    u = fu.get(level)
    n = (1 << (level + 1)) + 1
    npoints = n * (n + 1) * (n + 2) // 6
    err = np.sqrt(np.sum((u - exact) ** 2) / npoints)
    assert err < target, f"discrete L2 error {err:.3e} >= {target:.1e} (level {level}, {it} CG iterations)"
    uo = u0.copy()
    orc.cg(uo, f, level, tol=1e-12, max_iter=1000, op=orc.op_divkgrad_callback(1))
    close(u, uo, 1e-9)


def test_host_callback_quadrature_matches_oracle_and_device_factors(cube):
    """Any coefficient callback, evaluated on the host at every micro-tet's quadrature points
    (hyb_operator_create_divkgrad_callback_quadrature): with tanh(2 (x - 1/2)) + 2 its apply
    matches the oracle's callback operator (1e-12) and the device-evaluated kind 1 (1e-13)."""
    H, st, orc, L, w, ph = cube
    A = H.P1ElementwiseDivKGradOperator.callback_quadrature(st, 0, L, lambda p: np.tanh(2.0 * (p[0] - 0.5)) + 2.0)
    Ad = H.P1ElementwiseDivKGradOperator.quadrature(st, 0, L, 1)
    op = orc.op_divkgrad_callback(1)
    rng = np.random.default_rng(41)
    for level in range(L + 1):
        x = rng.uniform(-1, 1, orc.n(level))
        fs, fd, fe = (H.P1Function(n, st, 0, L) for n in "sde")
        fs.set(x, level)
        A.apply(fs, fd, level, H.ALL)
        Ad.apply(fs, fe, level, H.ALL)
        close(fd.get(level), orc.apply(x, level, flag=H.ALL, op=op), 1e-12)
        close(fd.get(level), fe.get(level), 1e-13)
