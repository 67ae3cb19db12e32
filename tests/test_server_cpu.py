"""Host-side logic of the serving loop (no GPU): request validation, footprint accounting,
budget refusal and the seeded coefficient features. Creating a server, sizing and
submitting requests make no device call, so these run on the CPU."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def H():
    import hyteg_b200 as H

    H.load()
    return H


def footprint_formula(nx, ny, nz, level, coeff, precision, mesh_max_level, modes=64, mesh=0):
    """Independent restatement of the per-request device bytes (the hierarchy's vectors per
    level, coefficient storage, coarse CG scratch, dot-product partials, features, the
    coarse-level program kernel's phase list)."""
    nC = 60 * (nx - 1) ** 2 * (ny - 1) if mesh == 1 else 6 * nx * ny * nz
    pad = lambda s: (s + 31) // 32 * 32
    closure = lambda l: ((1 << l) + 1) * ((1 << l) + 2) * ((1 << l) + 3) // 6
    per = 24 + (20 if precision == 32 else 0) + (12 if coeff != 0 else 0)
    b = sum(nC * pad(closure(l)) * per + (nC * 96 * 12 if coeff != 0 else 0) for l in range(level + 1))
    b += nC * pad(4) * 8 * (5 if precision == 32 else 3)
    b += max(-(-closure(l) // 256) * nC for l in range(mesh_max_level + 1)) * 8
    b += (level + 1) * 65536  # phase-list allowance of the coarse-level program kernel
    return b + 16 + 16 + 4 * modes * 8


@pytest.mark.parametrize("shape", [(1, 1, 1, 3, 0, 64), (2, 2, 2, 7, 1, 32), (4, 4, 4, 6, 1, 64), (3, 3, 3, 5, 0, 32)])
def test_footprint_matches_formula(H, shape):
    sv = H.Server(1 << 40, max_level=7)
    nx, ny, nz, L, coeff, prec = shape
    req = H.Server.request(nx, ny, nz, L, coeff, prec)
    assert sv.footprint(req) == footprint_formula(nx, ny, nz, L, coeff, prec, 7)


@pytest.mark.parametrize("shape", [(5, 4, 6, 2, 32), (3, 2, 3, 0, 64)])
def test_shell_footprint_matches_formula(H, shape):
    sv = H.Server(1 << 40, max_level=7)
    ntan, nrad, L, coeff, prec = shape
    req = H.Server.request(ntan, nrad, 1, L, coeff, prec, mesh=H.MESH_SHELL)
    assert sv.footprint(req) == footprint_formula(ntan, nrad, 1, L, coeff, prec, 7, mesh=1)


def test_invalid_requests_are_refused(H):
    sv = H.Server(1 << 40, max_level=7)
    bad = [H.Server.request(0, 1, 1, 3), H.Server.request(1, 1, 1, 8), H.Server.request(1, 1, 1, 0),
           H.Server.request(1, 1, 1, 3, coefficient=5), H.Server.request(1, 1, 1, 3, precision=16),
           H.Server.request(1, 1, 1, 3, rel_tol=0.0), H.Server.request(1, 1, 1, 3, max_cycles=0),
           H.Server.request(1, 1, 1, 3, rel_tol=float("nan")), H.Server.request(1, 1, 1, 3, mesh=7),
           H.Server.request(1, 2, 1, 3, mesh=H.MESH_SHELL), H.Server.request(1, 1, 1, 3, coefficient=3)]
    for req in bad:
        with pytest.raises(H.HybError, match="error 1:"):
            sv.submit(req)
    with pytest.raises(H.HybError, match="arrival"):
        sv.submit(H.Server.request(1, 1, 1, 3), arrival_s=-1.0)


def test_oversized_request_is_refused_with_enomem(H):
    req = H.Server.request(4, 4, 4, 7, 1, 32)
    sv = H.Server(1 << 30, max_level=7)  # 1 GiB: a level-7 4x4x4 hierarchy needs several
    need = sv.footprint(req)
    assert need > 1 << 30
    with pytest.raises(H.HybError, match="error 2:.*more than the budget"):
        sv.submit(req)
    small = H.Server.request(1, 1, 1, 3)
    assert sv.submit(small) == 0  # the refused one was not queued


def test_server_arguments_validated(H):
    for args in [(0, 4, 7), (1 << 30, 0, 7), (1 << 30, 4, 0), (1 << 30, 4, 10)]:
        with pytest.raises(H.HybError):
            H.Server(*args)


def test_rff_features_are_seeded_gaussian(H):
    w1, p1 = H.rff_features(3, 0.2, 64)
    w2, p2 = H.rff_features(3, 0.2, 64)
    w3, _ = H.rff_features(4, 0.2, 64)
    assert np.array_equal(w1, w2) and np.array_equal(p1, p2)
    assert not np.array_equal(w1, w3)
    assert np.all((p1 >= 0) & (p1 < 2 * np.pi))
    # many draws: N(0, 1/0.2^2) components and U[0, 2 pi) phases
    w, p = H.rff_features(11, 0.2, 4096)
    assert abs(w.mean()) < 0.2 and abs(w.std() - 5.0) < 0.2
    assert abs(p.mean() - np.pi) < 0.1
