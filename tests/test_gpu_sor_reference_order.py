"""The SOR sweep in the reference's own order (hyb_operator_smooth_sor_reference_order):
macro-vertices, -edges, -faces, then -cells (backwards: the reverse, with the ghost layers
refreshed between stages), each primitive lexicographic and reading only its own closure's
current values (P1Operator.hpp:352-431). On the GPU each stage computes the affine part of
every point's update at once and then walks the edge's points, the face's hyperplanes
i + 2j and the cell's hyperplanes x + 2y + 3z over on-chip memory (k_sorref_edges_fast,
k_sorref_faces_pre/_stage, k_sorref_cells_pre/_stage/_scatter); the plain walks
(k_sorref_edges/_faces/_cells) run the cells of coefficient operators, the stages whose
shared memory would not fit, and everything under HYB_SORREF_SIMPLE=1 (tested in a
subprocess). Checked against the oracle's reference-order
sweep, whose face stage is pinned to the generated macro-face kernels: one sweep 1e-11 (the
multicolour sweep's tolerance), also at level 7 on the benchmarked 48-tet mesh; FP32 1e-5;
V(3,3) cycles with the forward and the symmetric smoother 1e-10 against the oracle's cycles
with smoother 0 and 3."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def close(a, b, rtol):
    err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    assert err <= rtol, f"max relative error {err:.3e} > {rtol:.1e}"


@pytest.fixture(scope="module")
def setups(oracle_mod):
    import hyteg_b200 as H

    H.load()
    O = oracle_mod
    g = np.load(os.path.join(GOLD, "reference_meshes.npz"))
    out = {}
    L = 4
    for name, (c, t) in {
        "cube211": O.mesh_cuboid(2, 1, 1, hi=(2.0, 1.0, 1.0)),
        "octahedron": (g["regular_octahedron_8el_coords"], g["regular_octahedron_8el_tets"]),
        "tet_1el": (g["tet_1el_coords"], g["tet_1el_tets"]),
    }.items():
        out[name] = (H.PrimitiveStorage(c, t, L), O.Oracle(c, t, L), L)
    return H, O, out


def operators(H, O, st, orc, L, kind):
    if kind == "laplace":
        return H.P1ConstantLaplaceOperator(st, 0, L), 0
    if kind == "nodal":
        kv = [O.grf_coefficient(orc.coords_of(l), seed=3) for l in range(L + 1)]
        return H.P1ElementwiseDivKGradOperator(st, 0, L, kv), orc.op_divkgrad(kv)
    return H.P1ElementwiseDivKGradOperator.quadrature(st, 0, L, 1), orc.op_divkgrad_callback(1)


@pytest.mark.parametrize("name", ["cube211", "octahedron", "tet_1el"])
@pytest.mark.parametrize("kind", ["laplace", "nodal", "quadrature"])
def test_one_sweep_matches_oracle(setups, name, kind):
    H, O, S = setups
    st, orc, L = S[name]
    A, op = operators(H, O, st, orc, L, kind)
    rng = np.random.default_rng(17)
    for level in range(L + 1):
        for flag in (H.INNER | H.NEUMANN, H.ALL):
            for backwards in (False, True):
                for relax in (1.0, 0.8):
                    x, b = rng.uniform(-1, 1, orc.n(level)), rng.uniform(-1, 1, orc.n(level))
                    fu, fb = H.P1Function("u", st, 0, L), H.P1Function("b", st, 0, L)
                    fu.set(x, level)
                    fb.set(b, level)
                    A.smooth_sor_reference_order(fu, fb, relax, level, flag, backwards=backwards)
                    xr = orc.sor_ref(x.copy(), b, level, relax=relax, flag=flag, op=op, backwards=backwards)
                    close(fu.get(level), xr, 1e-11)
                    # nothing outside flag moves
                    _, bc = orc.info(level)
                    fixed = (bc & flag) == 0
                    assert np.array_equal(fu.get(level)[fixed], x[fixed])


def test_differs_from_multicolour_order(setups):
    """The two orders are different sweeps: on the same inputs they give different iterates
    (the check above is not passing on a sweep that ignores the order)."""
    H, O, S = setups
    st, orc, L = S["cube211"]
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    rng = np.random.default_rng(5)
    x, b = rng.uniform(-1, 1, orc.n(L)), rng.uniform(-1, 1, orc.n(L))
    f1, f2, fb = (H.P1Function(n, st, 0, L) for n in ("u1", "u2", "b"))
    for f in (f1, f2):
        f.set(x, L)
    fb.set(b, L)
    A.smooth_sor_reference_order(f1, fb, 1.0, L, H.INNER | H.NEUMANN)
    A.smooth_sor(f2, fb, 1.0, L, H.INNER | H.NEUMANN)
    assert np.abs(f1.get(L) - f2.get(L)).max() > 1e-3


def test_fp32_sweep(setups):
    H, O, S = setups
    st, orc, L = S["cube211"]
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    rng = np.random.default_rng(23)
    x, b = rng.uniform(-1, 1, orc.n(L)), rng.uniform(-1, 1, orc.n(L))
    fu, fb = H.P1Function("u", st, 0, L, H.F32), H.P1Function("b", st, 0, L, H.F32)
    fu.set(x.astype(np.float32), L)
    fb.set(b.astype(np.float32), L)
    for backwards in (False, True):
        A.smooth_sor_reference_order(fu, fb, 1.0, L, H.INNER | H.NEUMANN, backwards=backwards)
    xr = orc.sor_ref(x.astype(np.float32).astype(np.float64), b.astype(np.float32).astype(np.float64), L)
    xr = orc.sor_ref(xr, b.astype(np.float32).astype(np.float64), L, backwards=True)
    close(fu.get(L).astype(np.float64), xr, 1e-5)


@pytest.mark.parametrize("smoother,oracle_smoother", [(4, 0), (5, 3)])
@pytest.mark.parametrize("kind", ["laplace", "nodal"])
def test_vcycles_match_oracle(setups, smoother, oracle_smoother, kind):
    """GeometricMultigridSolver with SORSmoother / SymmetricSORSmoother in the reference's
    order: two V(3,3) cycles equal the oracle's reference-order cycles (1e-10), and the
    solve to 1e-8 takes the oracle's cycle count."""
    H, O, S = setups
    st, orc, L = S["cube211"]
    A, op = operators(H, O, st, orc, L, kind)
    b = O.uniform_rhs(orc.coords_of(L), 3, 2 << L)
    fx, fb = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
    fx.set(np.zeros(orc.n(L)), L)
    fb.set(b, L)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0, smoother=smoother, coarse_tol=1e-14)
    x = np.zeros(orc.n(L))
    for _ in range(2):
        gmg.solve(fx, fb, L)
        fb.set(b, L)
        orc.gmg(x, b, 0, L, pre=3, post=3, relax=1.0, smoother=oracle_smoother, coarse_tol=1e-14, max_cycles=1, op=op)
        close(fx.get(L), x, 1e-10)
    fx.set(np.zeros(orc.n(L)), L)
    hist = gmg.solve_to_tolerance(fx, fb, L, 1e-8, max_cycles=60)
    _, h_ref = orc.gmg(np.zeros(orc.n(L)), b, 0, L, pre=3, post=3, smoother=oracle_smoother, coarse_tol=1e-14,
                       max_cycles=60, rel_tol=1e-8, op=op)
    assert len(hist) == len(h_ref), (hist, h_ref)
    close(np.asarray(hist), np.asarray(h_ref), 1e-6)


def test_level7_cube48_sweeps(setups, oracle_mod):
    """Forward then backward sweep on the 2x2x2 cuboid at level 7 (16.97 M DoFs; the face
    wavefront takes 64 KB of shared memory, the cell ring 44 KB)."""
    H, O, _ = setups
    c, t = O.mesh_cuboid(2, 2, 2)
    L = 7
    st, orc = H.PrimitiveStorage(c, t, L), O.Oracle(c, t, L)
    A = H.P1ConstantLaplaceOperator(st, L, L)
    rng = np.random.default_rng(29)
    x, b = rng.uniform(-1, 1, orc.n(L)), rng.uniform(-1, 1, orc.n(L))
    fu, fb = H.P1Function("u", st, L, L), H.P1Function("b", st, L, L)
    fu.set(x, L)
    fb.set(b, L)
    for backwards in (False, True):
        A.smooth_sor_reference_order(fu, fb, 1.0, L, H.INNER | H.NEUMANN, backwards=backwards)
        orc.sor_ref(x, b, L, backwards=backwards)
        close(fu.get(L), x, 1e-11)


def test_mixed_precision_solve(setups):
    """The mixed-precision solver with the reference-order smoother (FP32 sweeps) reaches 1e-8
    and agrees with the oracle's tightly converged FP64 solution to 1e-6."""
    H, O, S = setups
    st, orc, L = S["cube211"]
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    b = O.uniform_rhs(orc.coords_of(L), 3, 2 << L)
    fx, fb = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
    fb.set(b, L)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0, smoother=H.SMOOTHER_SOR_REFERENCE_ORDER)
    hist = gmg.solve_to_tolerance(fx, fb, L, 1e-8, max_cycles=60, precision=32)
    assert hist[-1] <= 1e-8
    xr = np.zeros(orc.n(L))
    orc.gmg(xr, b, 0, L, pre=3, post=3, smoother=0, max_cycles=100, rel_tol=1e-13)
    close(fx.get(L), xr, 1e-6)


def _simple_errors():
    """The plain hyperplane kernels (HYB_SORREF_SIMPLE=1): sweeps on the 2x1x1 cuboid at
    levels 3 and 4, Laplacian and nodal coefficient, both directions; prints the errors."""
    import hyteg_b200 as H
    import oracle as O

    H.load()
    L = 4
    c, t = O.mesh_cuboid(2, 1, 1, hi=(2.0, 1.0, 1.0))
    st, orc = H.PrimitiveStorage(c, t, L), O.Oracle(c, t, L)
    errs = {}
    rng = np.random.default_rng(37)
    for kind in ("laplace", "nodal"):
        A, op = operators(H, O, st, orc, L, kind)
        for level in (3, 4):
            for backwards in (False, True):
                x, b = rng.uniform(-1, 1, orc.n(level)), rng.uniform(-1, 1, orc.n(level))
                fu, fb = H.P1Function("u", st, 0, L), H.P1Function("b", st, 0, L)
                fu.set(x, level)
                fb.set(b, level)
                A.smooth_sor_reference_order(fu, fb, 0.8, level, H.ALL, backwards=backwards)
                xr = orc.sor_ref(x.copy(), b, level, relax=0.8, flag=H.ALL, op=op, backwards=backwards)
                errs[f"{kind}_L{level}_bw{int(backwards)}"] = float(np.abs(fu.get(level) - xr).max() /
                                                                    np.abs(xr).max())
    print("SIMPLE_ERRORS " + json.dumps(errs))


def test_plain_walk_kernels_in_subprocess():
    env = dict(os.environ, HYB_SORREF_SIMPLE="1")
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--simple-errors"], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("SIMPLE_ERRORS ")][-1]
    for k, e in json.loads(line.split(" ", 1)[1]).items():
        assert e <= 1e-11, f"{k}: {e:.3e}"


if __name__ == "__main__" and "--simple-errors" in sys.argv:
    for sub in ("oracle", os.path.join("hyteg-vara_b200", "python")):
        sys.path.insert(0, os.path.join(ROOT, sub))
    _simple_errors()


def test_level8_single_tet_fp32_ring_walk(setups, oracle_mod):
    """FP32 at level 8 on one macro-tet: the face interior and its staged couplings fit shared
    memory (k_sorref_faces_stage), the cell walk's ring fits but its staging does not, so the
    cells run the ring walk with register prefetch (k_sorref_cells_wave). Forward then
    backward against the oracle's FP64 sweeps of the same FP32-rounded inputs (FP32
    tolerance 2e-5)."""
    H, O, _ = setups
    g = np.load(os.path.join(GOLD, "reference_meshes.npz"))
    c, t = g["tet_1el_coords"], g["tet_1el_tets"]
    L = 8
    st, orc = H.PrimitiveStorage(c, t, L), O.Oracle(c, t, L)
    A = H.P1ConstantLaplaceOperator(st, L, L)
    rng = np.random.default_rng(43)
    x = rng.uniform(-1, 1, orc.n(L)).astype(np.float32).astype(np.float64)
    b = rng.uniform(-1, 1, orc.n(L)).astype(np.float32).astype(np.float64)
    fu, fb = H.P1Function("u", st, L, L, H.F32), H.P1Function("b", st, L, L, H.F32)
    fu.set(x.astype(np.float32), L)
    fb.set(b.astype(np.float32), L)
    for backwards in (False, True):
        A.smooth_sor_reference_order(fu, fb, 1.0, L, H.INNER | H.NEUMANN, backwards=backwards)
        orc.sor_ref(x, b, L, backwards=backwards)
        close(fu.get(L).astype(np.float64), x, 2e-5)
