"""Stage timers of the multigrid solver in the shape of the reference's timing tree
(GeometricMultigridSolver.hpp:129-233): node names, nesting and counts after a few
V-cycles, consistent totals, and the same iterate as an untimed solver (1e-12, the
tolerance of the other V-cycle tests)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def H():
    import hyteg_b200 as H

    H.load()
    return H


def rel_diff(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_timing_tree_shape_counts_and_unchanged_result(H):
    L, pre, post, cycles = 5, 2, 2, 3
    st = H.PrimitiveStorage.cuboid(1, 1, 1, L)
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    b = H.P1Function("b", st, 0, L)
    b.fill_uniform_random(L, 3, float(1 << L))
    x0, x1 = H.P1Function("x0", st, 0, L), H.P1Function("x1", st, 0, L)
    plain = H.GeometricMultigridSolver(st, A, 0, L, pre, post, 1.0)
    timed = H.GeometricMultigridSolver(st, A, 0, L, pre, post, 1.0)
    timed.set_timing(True)
    b1 = H.P1Function("b1", st, 0, L)  # the V-cycle uses b's coarse levels as scratch
    b1.fill_uniform_random(L, 3, float(1 << L))
    for _ in range(cycles):
        plain.solve(x0, b, L)
        timed.solve(x1, b1, L)
    assert rel_diff(x1.get(L), x0.get(L)) <= 1e-12

    t = timed.timing()
    assert list(t) == ["Geometric Multigrid Solver"]
    gms = t["Geometric Multigrid Solver"]
    assert gms["count"] == cycles and gms["total"] > 0
    levels = gms["children"]
    assert set(levels) == {f"Level {l}" for l in range(L + 1)}
    for l in range(1, L + 1):
        node = levels[f"Level {l}"]
        assert node["count"] == 2 * cycles  # before and after the coarse-grid correction
        kids = node["children"]
        assert set(kids) == {"Smoother", "Restriction", "Prolongation"}
        assert kids["Smoother"]["count"] == (pre + post) * cycles
        assert kids["Restriction"]["count"] == cycles and kids["Prolongation"]["count"] == cycles
        assert sum(k["total"] for k in kids.values()) <= node["total"] * 1.001 + 1e-6
        for k in kids.values():
            assert 0 < k["min"] <= k["average"] <= k["max"]
    coarse = levels["Level 0"]
    assert coarse["count"] == cycles and list(coarse["children"]) == ["Coarse Grid Solver"]
    assert sum(v["total"] for v in levels.values()) <= gms["total"] * 1.001 + 1e-6

    timed.reset_timing()
    assert timed.timing() == {}


def test_timing_tree_mixed_precision_solve(H):
    """solve_to_tolerance with FP32 cycles: one "Geometric Multigrid Solver" node per
    refinement step, and the residual history of the untimed solver. With the timers on,
    the levels the one-block program kernel would run are launched one by one, whose FP32
    sums can round differently. The differences start at FP32 rounding (4e-8 relative in
    the first step) and grow over the steps to about 1e-6, so the histories must agree to
    1e-5 relative, with the same number of steps."""
    L = 4
    st = H.PrimitiveStorage.cuboid(1, 1, 1, L)
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    hists = []
    for timing in (False, True):
        x, b = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
        b.fill_uniform_random(L, 5, float(1 << L))
        g = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0)
        g.set_timing(timing)
        hists.append(g.solve_to_tolerance(x, b, L, 1e-8, max_cycles=50, precision=32))
        if timing:
            t = g.timing()
            assert t["Geometric Multigrid Solver"]["count"] == len(hists[-1]) - 1
    assert len(hists[0]) == len(hists[1])
    assert np.allclose(hists[0], hists[1], rtol=1e-5, atol=0)
