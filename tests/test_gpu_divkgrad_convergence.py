"""The reference's ElementwiseDivKGradCGConvergenceTest (P1 part, 3D;
tests/hyteg/convergence/ElementwiseDivKGradCGConvergenceTest.cpp:41-137) restated through the
GPU variable-coefficient operator and the GPU CG:

  -div(k grad u) = f on the reference's one-tetrahedron mesh (data/meshes/3D/tet_1el.msh),
  exact u = sin(phi pi x) sinh(pi y), k = tanh(alpha (x - 1/2)) + 2, alpha = phi = 2;
  f = M r with r the interpolated right-hand side and M the P1 mass matrix (the oracle's
  P1ElementwiseMassOperator supplies it); u = exact on the Dirichlet boundary; CG to 1e-12,
  at most 1000 iterations; discrete L2 error sqrt(sum (u - u_exact)^2 / npoints) with npoints
  the number of P2 DoFs of the level, as the reference computes it.

Thresholds are the reference's: 1.1e-3 (level 3), 3.5e-4 (level 4), 1.0e-4 (level 5). The
coefficient enters the GPU operator through its nodal values (the P1 interpolant), where the
reference form evaluates the callback at its quadrature points; the errors stay below the
same thresholds."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.mark.parametrize("level,target", [(3, 1.1e-3), (4, 3.5e-4), (5, 1.0e-4)])
def test_divkgrad_cg_convergence_tet_1el(oracle_mod, level, target):
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
    k = np.tanh(alpha * (x - 0.5)) + 2.0
    t0 = np.tanh(alpha * (x - 0.5))
    t1 = phi * alpha * (t0 * t0 - 1.0) * np.cos(phi * np.pi * x)
    t2 = (phi * phi - 1.0) * np.pi * (t0 + 2.0) * np.sin(phi * np.pi * x)
    r = np.pi * (t1 + t2) * np.sinh(np.pi * y)
    f = orc.apply(r, level, flag=O.ALL, op=orc.op_mass())
    kind, bc = orc.info(level)
    u0 = np.where((bc & O.DIRICHLET) != 0, exact, 0.0)
    A = H.P1ElementwiseDivKGradOperator(st, level, level, [k])
    fu, ff = H.P1Function("u", st, level, level), H.P1Function("f", st, level, level)
    fu.set(u0, level)
    ff.set(f, level)
    it, conv = H.CGSolver(tolerance=1e-12, max_iter=1000).solve(A, fu, ff, level)
    u = fu.get(level)
    n = (1 << (level + 1)) + 1
    npoints = n * (n + 1) * (n + 2) // 6  # P2 DoFs of the level = P1 DoFs one level up
    err = np.sqrt(np.sum((u - exact) ** 2) / npoints)
    assert err < target, f"discrete L2 error {err:.3e} >= {target:.1e} (level {level}, {it} CG iterations)"
