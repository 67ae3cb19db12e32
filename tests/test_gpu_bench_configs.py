"""GPU parity at the benchmarked sizes, through the C ABI, against the CPU oracle.

The small-mesh parity tests run every operation at level <= 5 on meshes of at most six
macro-tets, where the large-level kernel paths never run. These tests run the paths the
benchmarks time, on the benchmarked meshes and levels:

* Poisson on the 2x2x2 cuboid (48 macro-tets) at level 7 (16,974,593 DoFs): the constant
  apply (interior quads + surface lane groups, ``k_apply``), one multicolour SOR sweep
  (surface lane groups ``k_sor_iface`` -- the level is above the row-table bounds -- then
  the per-colour interior passes ``k_sor_interior``) in FP64 and FP32, and one V(3,3)
  cycle over levels 0..7 (program kernel, row passes, launched levels);
* -div(k grad u) on the 4x4x4 cuboid (384 macro-tets) at level 6 with k = exp(g), g the
  seeded Gaussian random field (correlation length 0.2, sigma 1): the variable-coefficient
  apply and SOR sweep (``k_apply<VAR>``, ``k_sor_iface<VAR>``, ``k_sor_interior<VAR>``);
* every kernel branch that the environment thresholds HYB_ROW_TABLE_MAX_POINTS,
  HYB_ROW_IFACE_MAX_POINTS, HYB_FUSED_INTERIOR_MAX and HYB_PROGRAM_MAX_POINTS select,
  forced in a subprocess and checked against the same oracle results.

Tolerances (max-norm, relative to the oracle's result): apply 1e-12, FP64 SOR sweep 1e-11,
V-cycle 1e-10; the FP32 sweep (FP32 inputs, FP32 arithmetic) against the oracle's FP64
sweep of the same FP32-rounded inputs: 2e-5.

Reference: src/hyteg/p1functionspace/generatedKernels/sor_3D_macrocell_P1.cpp:31-77,
src/hyteg/p1functionspace/P1Operator.hpp:196-324, 352-422.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for sub in ("oracle", os.path.join("hyteg-vara_b200", "python")):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-300))


def close(a, b, rtol):
    err = rel_err(a, b)
    assert err <= rtol, f"max relative error {err:.3e} > {rtol:.1e}"


@pytest.fixture(scope="module")
def H():
    import hyteg_b200 as H

    H.load()
    return H


@pytest.fixture(scope="module")
def cube48(H, oracle_mod):
    """The 2x2x2 cuboid at level 7 (GPU storage and oracle)."""
    O = oracle_mod
    L = 7
    c, t = O.mesh_cuboid(2, 2, 2)
    assert len(t) == 48
    st = H.PrimitiveStorage(c, t, L)
    orc = O.Oracle(c, t, L)
    assert st.num_dofs(L) == orc.n(L) == 257 ** 3
    return st, orc, L


def test_level7_cube48_apply(H, cube48):
    """k_apply<double, constant, replace/add> on 16.97 M DoFs: interior quads and surface
    lane groups, flags Inner and All."""
    st, orc, L = cube48
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, orc.n(L))
    y0 = rng.uniform(-1, 1, orc.n(L))
    fs, fd = H.P1Function("s", st, L, L), H.P1Function("d", st, L, L)
    fs.set(x, L)
    for flag, update in ((H.INNER, H.REPLACE), (H.ALL, H.ADD)):
        fd.set(y0, L)
        A.apply(fs, fd, L, flag, update)
        ref = orc.apply(x, L, flag=flag, dst=y0.copy(), add=bool(update))
        close(fd.get(L), ref, 1e-12)


def test_level7_cube48_sor_sweep_fp64(H, cube48):
    """One FP64 multicolour SOR sweep at level 7 (six surface passes k_sor_iface, four
    interior passes k_sor_interior), then a second one, against the oracle's identical
    multicolour order."""
    st, orc, L = cube48
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    m, labels = st.colouring()
    rng = np.random.default_rng(12)
    x, b = rng.uniform(-1, 1, orc.n(L)), rng.uniform(-1, 1, orc.n(L))
    fx, fb = H.P1Function("x", st, L, L), H.P1Function("b", st, L, L)
    fx.set(x, L)
    fb.set(b, L)
    for _ in range(2):
        A.smooth_sor(fx, fb, 1.0, L, H.INNER | H.NEUMANN)
        orc.sor_colored(x, b, L, labels, m, relax=1.0, flag=H.INNER | H.NEUMANN)
        close(fx.get(L), x, 1e-11)


def test_level7_cube48_sor_sweep_fp32(H, cube48):
    """The FP32 sweep of the mixed-precision V-cycles at level 7 against the oracle's FP64
    sweep of the same FP32-rounded inputs."""
    st, orc, L = cube48
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    m, labels = st.colouring()
    rng = np.random.default_rng(13)
    x = rng.uniform(-1, 1, orc.n(L)).astype(np.float32)
    b = rng.uniform(-1, 1, orc.n(L)).astype(np.float32)
    fx, fb = H.P1Function("x", st, L, L, dtype=H.F32), H.P1Function("b", st, L, L, dtype=H.F32)
    fx.set(x, L)
    fb.set(b, L)
    A.smooth_sor(fx, fb, 1.0, L, H.INNER | H.NEUMANN)
    xr = x.astype(np.float64)
    orc.sor_colored(xr, b.astype(np.float64), L, labels, m, relax=1.0, flag=H.INNER | H.NEUMANN)
    close(fx.get(L), xr, 2e-5)


def test_level7_cube48_vcycle(H, oracle_mod, cube48):
    """One FP64 V(3,3) cycle over levels 0..7 (program kernel on levels 0-2, row passes on
    the middle levels, launched passes on levels 6-7) from a zero guess, f ~ U[-1, 1] seeded
    by lattice position, against the oracle's V-cycle with the same multicolour SOR."""
    O = oracle_mod
    st, orc, L = cube48
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    m, labels = st.colouring()
    b = O.uniform_rhs(orc.coords_of(L), 0, 2 << L)
    fx, fb = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
    fb.set(b, L)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0, coarse_tol=1e-14)
    gmg.solve(fx, fb, L)
    x = np.zeros(orc.n(L))
    orc.gmg(x, b, 0, L, pre=3, post=3, relax=1.0, smoother=1, labels=labels, m=m, coarse_tol=1e-14, max_cycles=1)
    close(fx.get(L), x, 1e-10)


@pytest.fixture(scope="module")
def cube384(H, oracle_mod):
    """The 4x4x4 cuboid at level 6 with the configuration's lognormal coefficient."""
    O = oracle_mod
    L = 6
    c, t = O.mesh_cuboid(4, 4, 4)
    assert len(t) == 384
    st = H.PrimitiveStorage(c, t, L)
    orc = O.Oracle(c, t, L)
    kv = [O.grf_coefficient(orc.coords_of(l), corr_len=0.2, sigma=1.0, seed=1) for l in range(L + 1)]
    A = H.P1ElementwiseDivKGradOperator(st, 0, L, kv)
    op = orc.op_divkgrad(kv)
    return st, orc, L, A, op


def test_level6_cube384_divkgrad_apply(H, cube384):
    """k_apply<double, variable> on 384 macro-tets at level 6 (16.97 M DoFs)."""
    st, orc, L, A, op = cube384
    rng = np.random.default_rng(14)
    x = rng.uniform(-1, 1, orc.n(L))
    fs, fd = H.P1Function("s", st, L, L), H.P1Function("d", st, L, L)
    fs.set(x, L)
    A.apply(fs, fd, L, H.ALL)
    close(fd.get(L), orc.apply(x, L, flag=H.ALL, op=op), 1e-12)


def test_level6_cube384_divkgrad_sor_sweep(H, cube384):
    """One FP64 variable-coefficient multicolour SOR sweep on 384 macro-tets at level 6."""
    st, orc, L, A, op = cube384
    m, labels = st.colouring()
    rng = np.random.default_rng(15)
    x, b = rng.uniform(-1, 1, orc.n(L)), rng.uniform(-1, 1, orc.n(L))
    fx, fb = H.P1Function("x", st, L, L), H.P1Function("b", st, L, L)
    fx.set(x, L)
    fb.set(b, L)
    A.smooth_sor(fx, fb, 1.0, L, H.INNER | H.NEUMANN)
    orc.sor_colored(x, b, L, labels, m, relax=1.0, flag=H.INNER | H.NEUMANN, op=op)
    close(fx.get(L), x, 1e-11)


# ---------------------------------------------------------------------------
# Environment-selected kernel branches, each forced in a fresh process
# ---------------------------------------------------------------------------
BIG = str(1 << 40)
BRANCHES = {
    # no row tables, per-colour interior launches on every level, no program kernel:
    # k_sor_iface / k_apply lane groups and k_sor_interior everywhere
    "lane_groups": {"HYB_ROW_TABLE_MAX_POINTS": "0", "HYB_ROW_IFACE_MAX_POINTS": "0",
                    "HYB_FUSED_INTERIOR_MAX": "0", "HYB_PROGRAM_MAX_POINTS": "0"},
    # full row tables (k_row_pass) on every level that has 16-bit row positions, the four
    # interior colours in one launch (k_sor_interior_cells) on every level
    "full_rows": {"HYB_ROW_TABLE_MAX_POINTS": BIG, "HYB_FUSED_INTERIOR_MAX": BIG},
    # rows of the surface colours only (k_row_pass surface + k_sor_interior)
    "surface_rows": {"HYB_ROW_TABLE_MAX_POINTS": "0", "HYB_ROW_IFACE_MAX_POINTS": BIG,
                     "HYB_FUSED_INTERIOR_MAX": "0"},
    # the program kernel on every level up to 4
    "program": {"HYB_PROGRAM_MAX_POINTS": "200000"},
}


def _branch_errors():
    """Apply, SOR sweep and one V-cycle on the 2x2x2 cuboid at level 5 and the variable-
    coefficient apply and sweep, each against the oracle; prints the errors as JSON."""
    import hyteg_b200 as H
    import oracle as O

    H.load()
    L = 5
    c, t = O.mesh_cuboid(2, 2, 2)
    st = H.PrimitiveStorage(c, t, L)
    orc = O.Oracle(c, t, L)
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    m, labels = st.colouring()
    rng = np.random.default_rng(21)
    errs = {}
    for level in (3, 4, 5):
        x, b = rng.uniform(-1, 1, orc.n(level)), rng.uniform(-1, 1, orc.n(level))
        fs, fd, fb = (H.P1Function(n, st, 0, L) for n in "sdb")
        fs.set(x, level)
        fb.set(b, level)
        A.apply(fs, fd, level, H.INNER | H.NEUMANN)
        errs[f"apply_L{level}"] = rel_err(fd.get(level), orc.apply(x, level, flag=H.INNER | H.NEUMANN))
        A.residual(fs, fb, fd, level, H.INNER | H.NEUMANN)
        kind, bc = orc.info(level)
        ax = orc.apply(x, level, flag=H.INNER | H.NEUMANN)
        errs[f"residual_L{level}"] = rel_err(fd.get(level), np.where((bc & 5) != 0, b - ax, 0.0))
        A.smooth_sor(fs, fb, 1.0, level, H.INNER | H.NEUMANN)
        A.smooth_sor_backwards(fs, fb, 1.0, level, H.INNER | H.NEUMANN)
        xr = orc.sor_colored(x.copy(), b, level, labels, m, flag=H.INNER | H.NEUMANN)
        xr = orc.sor_colored(xr, b, level, labels, m, flag=H.INNER | H.NEUMANN, backwards=True)
        errs[f"sor_fw_bw_L{level}"] = rel_err(fs.get(level), xr)
    bv = O.uniform_rhs(orc.coords_of(L), 0, 2 << L)
    fx, fb = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
    fb.set(bv, L)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0, coarse_tol=1e-14)
    gmg.solve(fx, fb, L)
    xr = np.zeros(orc.n(L))
    orc.gmg(xr, bv, 0, L, pre=3, post=3, smoother=1, labels=labels, m=m, coarse_tol=1e-14, max_cycles=1)
    errs["vcycle"] = rel_err(fx.get(L), xr)
    kv = [O.grf_coefficient(orc.coords_of(l), seed=1) for l in range(L + 1)]
    K = H.P1ElementwiseDivKGradOperator(st, 0, L, kv)
    op = orc.op_divkgrad(kv)
    x, b = rng.uniform(-1, 1, orc.n(L)), rng.uniform(-1, 1, orc.n(L))
    fs, fd, fb = (H.P1Function(n, st, 0, L) for n in "sdb")
    fs.set(x, L)
    fb.set(b, L)
    K.apply(fs, fd, L, H.ALL)
    errs["divkgrad_apply"] = rel_err(fd.get(L), orc.apply(x, L, flag=H.ALL, op=op))
    K.smooth_sor(fs, fb, 1.0, L, H.INNER | H.NEUMANN)
    errs["divkgrad_sor"] = rel_err(fs.get(L), orc.sor_colored(x.copy(), b, L, labels, m, flag=5, op=op))
    print("BRANCH_ERRORS " + json.dumps(errs))


@pytest.mark.parametrize("branch", sorted(BRANCHES))
def test_env_selected_kernel_branches(branch):
    env = dict(os.environ)
    env.update(BRANCHES[branch])
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--branch-errors"], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("BRANCH_ERRORS ")][-1]
    errs = json.loads(line.split(" ", 1)[1])
    tol = {"apply": 1e-12, "residual": 1e-12, "sor": 1e-11, "vcycle": 1e-10, "divkgrad_apply": 1e-12,
           "divkgrad_sor": 1e-11}
    for k, e in errs.items():
        t = tol.get(k) or tol[k.split("_")[0]]
        assert e <= t, f"{branch}: {k} error {e:.3e} > {t:.1e}"


if __name__ == "__main__" and "--branch-errors" in sys.argv:
    _branch_errors()
