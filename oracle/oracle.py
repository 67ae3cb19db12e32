"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference arm of bench.py, always as the checker or the timed
CPU baseline, never by the product path.

Also holds the synthetic-input definitions shared by tests and bench
(mesh generators restated from the reference, seeded right-hand sides and the
random-field coefficient), so GPU runs and oracle runs see identical inputs.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libhyteg_refkernels.so")

INNER, DIRICHLET, NEUMANN, FREESLIP, ALL = 1, 2, 4, 8, 15

_lib = None


def build(ref=False):
    """Compile the oracle (and, when the reference tree is present, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref and os.path.isdir("/root/reference/src"):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P, I, I64, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
        L.orc_create.restype = P
        L.orc_create.argtypes = [P, I64, P, I64, I]
        L.orc_destroy.argtypes = [P]
        L.orc_num_dofs.restype = I64
        L.orc_num_dofs.argtypes = [P, I]
        L.orc_num_prims.restype = I64
        L.orc_num_prims.argtypes = [P, I]
        L.orc_dof_coords.argtypes = [P, I, P]
        L.orc_dof_info.argtypes = [P, I, P, P]
        L.orc_cell_closure_map.argtypes = [P, I, I, P]
        L.orc_op_laplace.restype = I
        L.orc_op_laplace.argtypes = [P]
        L.orc_op_divkgrad.restype = I
        L.orc_op_divkgrad.argtypes = [P, P]
        L.orc_cell_stencil.argtypes = [P, I, I, I, I, P]
        L.orc_apply.argtypes = [P, I, I, P, P, I, I]
        L.orc_sor_ref.argtypes = [P, I, I, P, P, D, I]
        L.orc_sor_colored.argtypes = [P, I, I, P, P, D, I, P, I]
        L.orc_jacobi.argtypes = [P, I, I, P, P, D, I]
        L.orc_prolongate.argtypes = [P, I, P, P, I, I]
        L.orc_restrict.argtypes = [P, I, P, P, I]
        L.orc_dot.restype = D
        L.orc_dot.argtypes = [P, I, P, P, I]
        L.orc_cg.restype = I
        L.orc_cg.argtypes = [P, I, I, P, P, D, I]
        L.orc_gmg_solve.restype = I
        L.orc_gmg_solve.argtypes = [P, I, I, I, P, P, I, I, D, I, P, I, D, I, D, I, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """Macro-mesh + level hierarchy on the CPU (one value per unique micro-vertex)."""

    def __init__(self, coords, tets, max_level):
        self.coords = np.ascontiguousarray(coords, dtype=np.float64)
        self.tets = np.ascontiguousarray(tets, dtype=np.int64)
        self.max_level = max_level
        self.h = lib().orc_create(_p(self.coords), len(self.coords), _p(self.tets), len(self.tets), max_level)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def n(self, level):
        return int(lib().orc_num_dofs(self.h, level))

    def coords_of(self, level):
        out = np.zeros((self.n(level), 3))
        lib().orc_dof_coords(self.h, level, _p(out))
        return out

    def info(self, level):
        kind = np.zeros(self.n(level), np.uint8)
        bc = np.zeros(self.n(level), np.uint8)
        lib().orc_dof_info(self.h, level, _p(kind), _p(bc))
        return kind, bc

    def num_prims(self, kind):
        return int(lib().orc_num_prims(self.h, kind))

    def op_divkgrad(self, nodal_k):
        arrs = [np.ascontiguousarray(k, dtype=np.float64) for k in nodal_k]
        self._keep = arrs
        ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        return int(lib().orc_op_divkgrad(self.h, ptrs))

    def cell_stencil(self, level, cell, mask=0, op=0):
        out = np.zeros(15)
        lib().orc_cell_stencil(self.h, op, level, cell, mask, _p(out))
        return out

    def apply(self, src, level, flag=INNER | NEUMANN, dst=None, add=False, op=0):
        src = np.ascontiguousarray(src, dtype=np.float64)
        dst = np.zeros_like(src) if dst is None else dst
        lib().orc_apply(self.h, op, level, _p(src), _p(dst), flag, int(add))
        return dst

    def sor_ref(self, x, b, level, relax=1.0, flag=INNER | NEUMANN, op=0):
        lib().orc_sor_ref(self.h, op, level, _p(x), _p(np.ascontiguousarray(b, np.float64)), relax, flag)
        return x

    def sor_colored(self, x, b, level, labels, m, relax=1.0, flag=INNER | NEUMANN, op=0):
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        lib().orc_sor_colored(self.h, op, level, _p(x), _p(np.ascontiguousarray(b, np.float64)), relax, flag,
                              _p(lab), m)
        return x

    def jacobi(self, x, b, level, relax=1.0, flag=INNER | NEUMANN, op=0):
        lib().orc_jacobi(self.h, op, level, _p(x), _p(np.ascontiguousarray(b, np.float64)), relax, flag)
        return x

    def prolongate(self, coarse, coarse_level, fine=None, flag=INNER | NEUMANN, add=False):
        fine = np.zeros(self.n(coarse_level + 1)) if fine is None else fine
        lib().orc_prolongate(self.h, coarse_level, _p(np.ascontiguousarray(coarse, np.float64)), _p(fine), flag,
                             int(add))
        return fine

    def restrict(self, fine, fine_level, coarse=None, flag=INNER | NEUMANN):
        coarse = np.zeros(self.n(fine_level - 1)) if coarse is None else coarse
        lib().orc_restrict(self.h, fine_level, _p(np.ascontiguousarray(fine, np.float64)), _p(coarse), flag)
        return coarse

    def dot(self, a, b, level, flag=INNER | NEUMANN):
        return float(lib().orc_dot(self.h, level, _p(np.ascontiguousarray(a, np.float64)),
                                   _p(np.ascontiguousarray(b, np.float64)), flag))

    def cg(self, x, b, level, tol=1e-12, max_iter=100000, op=0):
        return int(lib().orc_cg(self.h, op, level, _p(x), _p(np.ascontiguousarray(b, np.float64)), tol, max_iter))

    def gmg(self, x, b, min_level, max_level, pre=3, post=3, relax=1.0, smoother=0, labels=None, m=0,
            coarse_tol=1e-12, max_cycles=10, rel_tol=0.0, precision=64, op=0):
        hist = np.zeros(max_cycles + 1)
        lab = np.ascontiguousarray(labels if labels is not None else np.zeros(1), dtype=np.int32)
        cyc = lib().orc_gmg_solve(self.h, op, min_level, max_level, _p(x), _p(np.ascontiguousarray(b, np.float64)),
                                  pre, post, relax, smoother, _p(lab), m, coarse_tol, max_cycles, rel_tol, precision,
                                  _p(hist))
        return x, hist[: cyc + 1]


# ---------------------------------------------------------------------------
# Reference kernels compiled from the reference tree (oracle/_ref), for pinning
# ---------------------------------------------------------------------------
_ref = None


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            return None
        R = ctypes.CDLL(REF_LIB)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        R.ref_apply_cell.argtypes = [P, P, I, P, I]
        R.ref_sor_cell.argtypes = [P, P, I, P, D, I]
        R.ref_prolongate_cell.argtypes = [P, P, I, P]
        R.ref_restrict_cell.argtypes = [P, P, I, P]
        R.ref_p1_tet_diffusion.argtypes = [P, P]
        _ref = R
    return _ref


# ---------------------------------------------------------------------------
# Synthetic inputs
# ---------------------------------------------------------------------------
def mesh_cuboid(nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """MeshInfo::meshCuboid (src/hyteg/mesh/MeshGenCuboid.cpp:34-160): vertices x-fastest,
    six tets per cube from the hexahedron table, cells in the std::map order of their
    vertex-id vectors (lexicographic), which is the order SetupPrimitiveStorage numbers them."""
    hx, hy, hz = [(hi[d] - lo[d]) / n for d, n in enumerate((nx, ny, nz))]
    coords = []
    for iz in range(nz + 1):
        for iy in range(ny + 1):
            for ix in range(nx + 1):
                coords.append((lo[0] + ix * hx, lo[1] + iy * hy, lo[2] + iz * hz))
    tnode = [(4, 5, 7, 3), (0, 3, 1, 4), (4, 1, 5, 3), (5, 6, 7, 2), (1, 3, 2, 5), (7, 2, 3, 5)]
    off = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    vid = lambda i, j, k: k * (nx + 1) * (ny + 1) + j * (nx + 1) + i
    tets = set()
    for iz in range(nz):
        for iy in range(ny):
            for ix in range(nx):
                for t in tnode:
                    tets.add(tuple(vid(ix + off[m][0], iy + off[m][1], iz + off[m][2]) for m in t))
    return np.array(coords, np.float64), np.array(sorted(tets), np.int64)


def splitmix64(x):
    """SplitMix64 finaliser on uint64 numpy arrays (counter-based, layout independent)."""
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    return z ^ (z >> np.uint64(31))


def uniform_rhs(xyz, seed, lattice):
    """f ~ U[-1,1] i.i.d. per micro-vertex, keyed by the vertex's integer position on the
    global lattice of spacing 1/lattice, so the value does not depend on memory layout."""
    key = np.rint(np.asarray(xyz) * lattice).astype(np.int64)
    k = (key[:, 0].astype(np.uint64) * np.uint64(1_000_003) + key[:, 1].astype(np.uint64)) * np.uint64(1_000_033) \
        + key[:, 2].astype(np.uint64)
    with np.errstate(over="ignore"):
        h = splitmix64(k ^ (np.uint64(seed) * np.uint64(0xD1B54A32D192ED03)))
    return (h >> np.uint64(11)).astype(np.float64) / float(1 << 53) * 2.0 - 1.0


def grf_coefficient(xyz, corr_len=0.2, sigma=1.0, seed=1, modes=64):
    """k = exp(g) with g a stationary Gaussian random field (squared-exponential covariance,
    correlation length corr_len, standard deviation sigma) drawn by random Fourier features."""
    rng = np.random.default_rng(seed)
    w = rng.normal(0.0, 1.0 / corr_len, size=(modes, 3))
    ph = rng.uniform(0.0, 2.0 * np.pi, size=modes)
    g = sigma * np.sqrt(2.0 / modes) * np.cos(np.asarray(xyz) @ w.T + ph).sum(axis=1)
    return np.exp(g)


def _closure_map(self, level, cell):
    N = 1 << level
    out = np.zeros((N + 1) * (N + 2) * (N + 3) // 6, np.int32)
    lib().orc_cell_closure_map(self.h, level, cell, _p(out))
    return out


Oracle.closure_map = _closure_map
