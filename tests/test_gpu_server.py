"""Serving loop on the GPU: each request's result is the same alone and in a mix of
concurrent requests (tolerance 1e-12 relative in the max norm; the kernels are
deterministic, so the solutions agree bit for bit in practice), equals the standalone
solver API on the same problem, meets its tolerance, and the loop respects its memory
budget and slot limit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def H():
    import hyteg_b200 as H

    H.load()
    return H


def ndofs(H, nx, ny, nz, level):
    st = H.PrimitiveStorage.cuboid(nx, ny, nz, level)
    return st.num_dofs(level)


def rel_diff(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def server_like_gmg(H, st, A, L):
    """The public solver configured as the server configures a hierarchy: a hierarchy whose
    finest level holds at most 65536 closure points runs whole V-cycles in the program kernel
    (HYB_PROGRAM_MAX_POINTS, read when a solver is created)."""
    import os

    old = os.environ.get("HYB_PROGRAM_MAX_POINTS")
    os.environ["HYB_PROGRAM_MAX_POINTS"] = "65536"
    try:
        return H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0)
    finally:
        if old is None:
            del os.environ["HYB_PROGRAM_MAX_POINTS"]
        else:
            os.environ["HYB_PROGRAM_MAX_POINTS"] = old


MIX = [  # (nx, ny, nz, level, coefficient, precision, seed)
    (2, 2, 2, 5, 1, 32, 3),  # the probe request
    (1, 1, 1, 6, 0, 32, 1),
    (2, 2, 2, 5, 1, 32, 4),  # same shape, other seed: a second hierarchy of that shape
    (3, 3, 3, 4, 0, 64, 5),
    (1, 1, 1, 3, 1, 64, 6),
    (2, 2, 2, 5, 0, 32, 7),
    (2, 2, 2, 5, 1, 32, 3),  # the probe again, later, on a reused hierarchy
]


def test_result_same_alone_and_in_mix(H):
    probe = MIX[0]
    n = ndofs(H, *probe[:4])
    alone = H.Server(8 << 30, max_active=8, max_level=6)
    rid = alone.submit(H.Server.request(*probe), keep_solution=True, num_dofs=n)
    alone.run(120)
    r = alone.result(rid)
    assert r.status == 0 and r.rel_residual <= 1e-8, (r.status, r.rel_residual)
    x_alone = alone.solution(rid)

    mix = H.Server(8 << 30, max_active=8, max_level=6)
    ids = []
    for i, q in enumerate(MIX):
        # the last one arrives after the first probe has finished and reuses its hierarchy
        # (the loop's clock starts before the first mesh is built, which takes about a second)
        arrival = 5.0 if i == len(MIX) - 1 else 0.002 * i
        ids.append(mix.submit(H.Server.request(*q), arrival_s=arrival, keep_solution=True,
                              num_dofs=ndofs(H, *q[:4])))
    mix.run(300)
    for i, q in zip(ids, MIX):
        res = mix.result(i)
        assert res.status == 0 and res.rel_residual <= 1e-8, (q, res.status, res.rel_residual)
        assert res.admit_s >= res.arrival_s and res.done_s >= res.admit_s
    for i in (ids[0], ids[-1]):
        assert mix.result(i).cycles == r.cycles
        assert rel_diff(mix.solution(i), x_alone) <= TOL
    # the mix really overlapped: some request was admitted before an earlier one finished
    res = [mix.result(i) for i in ids[:-1]]
    assert any(res[j].admit_s < res[j - 1].done_s for j in range(1, len(res)))
    st = mix.stats()
    assert st["hierarchies_built"] == 6  # the second probe reused a resident hierarchy
    assert st["peak_bytes"] <= 8 << 30


SMALL = [  # (nx, ny, nz, level, coefficient, precision, seed): whole V-cycles in the program kernel
    (1, 1, 1, 3, 0, 64, 11),
    (1, 1, 1, 4, 1, 64, 12),
    (1, 1, 1, 5, 0, 32, 13),
    (2, 2, 2, 4, 1, 32, 14),
    (2, 1, 1, 4, 0, 64, 15),
    (1, 2, 1, 3, 1, 32, 16),
]


def test_small_solves_batched_in_one_launch(H):
    """Small requests admitted together run as ONE batched whole-solve launch per operator
    kind (a thread block per solve, every cycle and stopping test on the device); each
    result equals the public solver's on the same problem: same cycle count, residual and
    solution within the tolerance of the other serving tests."""
    sv = H.Server(8 << 30, max_active=16, max_level=5)
    ids = [sv.submit(H.Server.request(*q), keep_solution=True, num_dofs=ndofs(H, *q[:4])) for q in SMALL]
    sv.run(300)
    st = sv.stats()
    assert st["batched_solves"] == len(SMALL)
    assert st["batches"] == 2  # constant and lognormal coefficients: one launch each
    for rid, (nx, ny, nz, L, coefficient, precision, seed) in zip(ids, SMALL):
        res = sv.result(rid)
        assert res.status == 0 and res.rel_residual <= 1e-8, (nx, ny, nz, L, res.status, res.rel_residual)
        storage = H.PrimitiveStorage.cuboid(nx, ny, nz, L)
        if coefficient:
            w, ph = H.rff_features(seed, 0.2, 64)
            A = H.P1ElementwiseDivKGradOperator.random_features(storage, 0, L, w, ph, 1.0)
        else:
            A = H.P1ConstantLaplaceOperator(storage, 0, L)
        x, b = H.P1Function("x", storage, 0, L), H.P1Function("b", storage, 0, L)
        b.fill_uniform_random(L, seed, float(np.lcm.reduce([nx, ny, nz]) << L))
        gmg = server_like_gmg(H, storage, A, L)
        hist = gmg.solve_to_tolerance(x, b, L, 1e-8, max_cycles=100, precision=precision)
        assert len(hist) - 1 == res.cycles, (nx, ny, nz, L)
        assert abs(hist[-1] - res.rel_residual) <= 1e-12 * max(hist[-1], 1e-300) + 1e-18
        assert rel_diff(sv.solution(rid), x.get(L)) <= TOL, (nx, ny, nz, L)


@pytest.mark.parametrize("coefficient", [0, 1])
def test_server_matches_standalone_solver(H, coefficient):
    """The same problem through the public solver API, configured as the server configures
    the hierarchy, gives the same solution."""
    nx, L, seed = 2, 4, 9
    sv = H.Server(4 << 30, max_level=L)
    n = ndofs(H, nx, nx, nx, L)
    rid = sv.submit(H.Server.request(nx, nx, nx, L, coefficient, 32, seed), keep_solution=True, num_dofs=n)
    sv.run(120)
    res = sv.result(rid)
    assert res.status == 0

    st = H.PrimitiveStorage.cuboid(nx, nx, nx, L)
    if coefficient:
        w, ph = H.rff_features(seed, 0.2, 64)
        A = H.P1ElementwiseDivKGradOperator.random_features(st, 0, L, w, ph, 1.0)
    else:
        A = H.P1ConstantLaplaceOperator(st, 0, L)
    x, b = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
    b.fill_uniform_random(L, seed, float(nx << L))
    gmg = server_like_gmg(H, st, A, L)
    hist = gmg.solve_to_tolerance(x, b, L, 1e-8, max_cycles=100, precision=32)
    assert len(hist) - 1 == res.cycles
    assert abs(hist[-1] - res.rel_residual) <= 1e-12 * max(hist[-1], 1e-300) + 1e-18
    assert rel_diff(sv.solution(rid), x.get(L)) <= TOL


def test_footprint_is_an_upper_bound(H):
    """The device bytes a resident hierarchy really holds never exceed its estimate, for the
    constant (row tables) and the lognormal coefficient, mixed and plain FP64."""
    reqs = [H.Server.request(*q) for q in [(2, 2, 2, 5, 0, 32, 1), (3, 3, 3, 4, 0, 64, 2), (1, 1, 1, 6, 0, 32, 3),
                                           (2, 2, 2, 5, 1, 32, 4), (2, 2, 2, 4, 1, 64, 5)]]
    sv = H.Server(8 << 30, max_active=8, max_level=6)
    ids = [sv.submit(q) for q in reqs]
    sv.run(120)
    for i, q in zip(ids, reqs):
        res = sv.result(i)
        assert res.status == 0, res.status
        assert 0 < res.footprint_bytes <= sv.footprint(q)


def test_footprint_bound_and_tight_budget(H):
    """A budget that holds one level-5 hierarchy at a time: requests wait for memory,
    idle hierarchies are evicted, and every request still completes. The shapes alternate
    between FP32-inner (the larger) and FP64 hierarchies, so that no two fit together."""
    reqs = [H.Server.request(2, 2, 2, 5, 1, p, s) for s, p in [(1, 32), (2, 64), (3, 32), (4, 64)]]
    probe = H.Server(1 << 40, max_level=5)
    need = max(probe.footprint(q) for q in reqs)
    probe.submit(reqs[1])
    probe.run(120)
    mesh = probe.stats()["mesh_bytes"]  # storage, Laplace operator and row tables of the mesh
    assert mesh > 0
    # room for the mesh and one hierarchy, not two
    budget = mesh + need + need // 2
    sv = H.Server(budget, max_active=4, max_level=5)
    ids = [sv.submit(q, arrival_s=0.0) for q in reqs]
    sv.run(120)
    for i, q in zip(ids, reqs):
        res = sv.result(i)
        assert res.status == 0, res.status
        assert 0 < res.footprint_bytes <= sv.footprint(q)
    st = sv.stats()
    assert st["peak_bytes"] <= budget
    # the first two can not both be resident: the second waited for the first to finish
    r0, r1 = sv.result(ids[0]), sv.result(ids[1])
    assert r1.admit_s >= r0.done_s


def test_not_converged_and_time_limit_status(H):
    sv = H.Server(4 << 30, max_level=5)
    a = sv.submit(H.Server.request(1, 1, 1, 5, 0, 64, 1, rel_tol=1e-30, max_cycles=2))
    sv.run(120)
    res = sv.result(a)
    assert res.status == 6 and res.cycles == 2  # HYB_ENOTCONVERGED after max_cycles


def test_shell_request_matches_standalone_solver(H):
    """A spherical-shell request with the radial coefficient gives the solution of the same
    problem built through the public API (shell storage, device coefficient with radial
    profile and sigma 0.5, right-hand side on the lattice 2^20)."""
    ntan, nrad, L, seed = 3, 2, 3, 21
    sv = H.Server(4 << 30, max_level=L)
    st = H.PrimitiveStorage.spherical_shell(ntan, nrad, 0.55, 1.0, L)
    n = st.num_dofs(L)
    req = H.Server.request(ntan, nrad, 1, L, H.COEFF_RADIAL, 32, seed, mesh=H.MESH_SHELL)
    rid = sv.submit(req, keep_solution=True, num_dofs=n)
    sv.run(120)
    res = sv.result(rid)
    assert res.status == 0 and res.rel_residual <= 1e-8
    w, ph = H.rff_features(seed, 0.2, 64)
    A = H.P1ElementwiseDivKGradOperator.random_features(st, 0, L, w, ph, 0.5, radial=5.0)
    x, b = H.P1Function("x", st, 0, L), H.P1Function("b", st, 0, L)
    b.fill_uniform_random(L, seed, float(1 << 20))
    gmg = server_like_gmg(H, st, A, L)
    hist = gmg.solve_to_tolerance(x, b, L, 1e-8, max_cycles=100, precision=32)
    assert len(hist) - 1 == res.cycles
    assert rel_diff(sv.solution(rid), x.get(L)) <= TOL
