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
REF_FACE_LIB = os.path.join(HERE, "_ref", "libhyteg_refface.so")

INNER, DIRICHLET, NEUMANN, FREESLIP, ALL = 1, 2, 4, 8, 15

_lib = None


def reference_root():
    """The reference checkout named by HYTEG_REFERENCE_ROOT, or None when it is unset or
    holds no source tree (the compiled reference pieces are then not built)."""
    root = os.environ.get("HYTEG_REFERENCE_ROOT")
    return root if root and os.path.isdir(os.path.join(root, "src")) else None


def build(ref=False):
    """Compile the oracle (and, when the reference tree is available, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    root = reference_root()
    if ref and root:
        jobs = str(max(1, min(8, os.cpu_count() or 1)))
        subprocess.run(["make", "-s", "-j", jobs, "-C", HERE, "ref", "REF_ROOT=" + root], check=True)


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
        L.orc_sor_ref.argtypes = [P, I, I, P, P, D, I, I]
        L.orc_sor_ref_stages.argtypes = [P, I, I, P, P, D, I, I, I]
        L.orc_apply_rows.argtypes = [P, I, I, P, P, I64, P]
        L.orc_sor_colored.argtypes = [P, I, I, P, P, D, I, P, I, I]
        L.orc_jacobi.argtypes = [P, I, I, P, P, D, I]
        L.orc_prolongate.argtypes = [P, I, P, P, I, I]
        L.orc_restrict.argtypes = [P, I, P, P, I]
        L.orc_dot.restype = D
        L.orc_dot.argtypes = [P, I, P, P, I]
        L.orc_cg.restype = I
        L.orc_cg.argtypes = [P, I, I, P, P, D, I]
        L.orc_chebyshev_coefficients.argtypes = [I, D, D, P]
        L.orc_set_chebyshev.argtypes = [P, I, D, D]
        L.orc_smooth_chebyshev.argtypes = [P, I, I, P, P]
        L.orc_inv_diag.argtypes = [P, I, I, P]
        L.orc_spectral_radius.restype = D
        L.orc_spectral_radius.argtypes = [P, I, I, I, P]
        L.orc_op_blend_div_k_grad.restype = I
        L.orc_op_blend_div_k_grad.argtypes = [P, D]
        L.orc_shell_map_eval.restype = I
        L.orc_shell_map_eval.argtypes = [P, I, P, P, P]
        L.orc_blend_element_matrix.restype = I
        L.orc_blend_element_matrix.argtypes = [P, I, P, D, P]
        L.orc_set_threads.restype = I
        L.orc_set_threads.argtypes = [I]
        L.orc_divkgrad_element_matrix.restype = I
        L.orc_divkgrad_element_matrix.argtypes = [P, I, P, P]
        L.orc_op_divkgrad_callback.restype = I
        L.orc_op_divkgrad_callback.argtypes = [P, I, P, P, I, D, D]
        L.orc_op_mass.restype = I
        L.orc_op_mass.argtypes = [P]
        L.orc_gmg_solve.restype = I
        L.orc_gmg_solve.argtypes = [P, I, I, I, P, P, I, I, D, I, P, I, D, I, D, I, P, I]
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

    def op_divkgrad_callback(self, kind, w=None, phase=None, sigma=1.0, radial=0.0):
        """The variable-coefficient operator as the reference assembles it: the coefficient
        evaluated as the form's callback at the quadrature points of every micro-tet on every
        level (kind 1: tanh(2 (x - 1/2)) + 2; kind 2: exp(radial (1 - |x|) + sigma sqrt(2/M)
        sum_m cos(w_m . x + phase_m)))."""
        w = np.ascontiguousarray(np.zeros((1, 3)) if w is None else w, np.float64).reshape(-1, 3)
        ph = np.ascontiguousarray(np.zeros(1) if phase is None else phase, np.float64).ravel()
        op = int(lib().orc_op_divkgrad_callback(self.h, int(kind), _p(w), _p(ph), len(ph), float(sigma),
                                                float(radial)))
        if op < 0:
            raise ValueError("unknown coefficient kind")
        return op

    def op_mass(self):
        """P1ElementwiseMassOperator (exact P1 mass matrix per micro-tet)."""
        return int(lib().orc_op_mass(self.h))

    def op_blend_div_k_grad(self, alpha=0.0):
        """P1ElementwiseBlendingDivKGradOperator on the cells' IcosahedralShellMaps,
        k(y) = exp(alpha (1 - |y|)) at the mapped quadrature points."""
        op = int(lib().orc_op_blend_div_k_grad(self.h, float(alpha)))
        if op < 0:
            raise ValueError("the mesh is not a spherical shell: a cell cannot be classified")
        return op

    def shell_map(self, cell, x):
        F, DF = np.zeros(3), np.zeros(9)
        xx = np.ascontiguousarray(x, dtype=np.float64)
        if lib().orc_shell_map_eval(self.h, cell, _p(xx), _p(F), _p(DF)) != 0:
            raise ValueError("the mesh is not a spherical shell")
        return F, DF.reshape(3, 3)

    def blend_element_matrix(self, cell, X, alpha=0.0):
        A = np.zeros(16)
        XX = np.ascontiguousarray(X, dtype=np.float64).reshape(12)
        if lib().orc_blend_element_matrix(self.h, cell, _p(XX), float(alpha), _p(A)) != 0:
            raise ValueError("the mesh is not a spherical shell")
        return A.reshape(4, 4)

    def cell_stencil(self, level, cell, mask=0, op=0):
        out = np.zeros(15)
        lib().orc_cell_stencil(self.h, op, level, cell, mask, _p(out))
        return out

    def apply(self, src, level, flag=INNER | NEUMANN, dst=None, add=False, op=0):
        src = np.ascontiguousarray(src, dtype=np.float64)
        dst = np.zeros_like(src) if dst is None else dst
        lib().orc_apply(self.h, op, level, _p(src), _p(dst), flag, int(add))
        return dst

    def apply_rows(self, src, level, dofs, op=0):
        """(A src) at the listed DoFs only."""
        src = np.ascontiguousarray(src, dtype=np.float64)
        dofs = np.ascontiguousarray(dofs, dtype=np.int64)
        out = np.zeros(len(dofs))
        lib().orc_apply_rows(self.h, op, level, _p(src), _p(dofs), len(dofs), _p(out))
        return out

    def sor_ref(self, x, b, level, relax=1.0, flag=INNER | NEUMANN, op=0, backwards=False, stages=15):
        """smooth_sor / smooth_sor_backwards; `stages` selects the primitive sweeps to run
        (bit 0 vertices, 1 edges, 2 faces, 3 cells)."""
        lib().orc_sor_ref_stages(self.h, op, level, _p(x), _p(np.ascontiguousarray(b, np.float64)), relax, flag,
                                 int(backwards), int(stages))
        return x

    def sor_colored(self, x, b, level, labels, m, relax=1.0, flag=INNER | NEUMANN, op=0, backwards=False):
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        lib().orc_sor_colored(self.h, op, level, _p(x), _p(np.ascontiguousarray(b, np.float64)), relax, flag,
                              _p(lab), m, int(backwards))
        return x

    def set_chebyshev(self, order, lower, upper):
        lib().orc_set_chebyshev(self.h, order, lower, upper)

    def smooth_chebyshev(self, x, b, level, op=0):
        lib().orc_smooth_chebyshev(self.h, op, level, _p(x), _p(np.ascontiguousarray(b, np.float64)))
        return x

    def inv_diag(self, level, op=0):
        out = np.zeros(self.n(level))
        lib().orc_inv_diag(self.h, op, level, _p(out))
        return out

    def spectral_radius(self, level, iterations, x, op=0):
        return lib().orc_spectral_radius(self.h, op, level, iterations, _p(x))

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
            coarse_tol=1e-12, max_cycles=10, rel_tol=0.0, precision=64, op=0, cycle="V"):
        """smoother: 0 reference-order SOR, 1 multicolour SOR, 2 weighted Jacobi, 3 and 4 their
        symmetric SOR counterparts (forward then backwards); cycle "V" or "W"."""
        hist = np.zeros(max_cycles + 1)
        lab = np.ascontiguousarray(labels if labels is not None else np.zeros(1), dtype=np.int32)
        cyc = lib().orc_gmg_solve(self.h, op, min_level, max_level, _p(x), _p(np.ascontiguousarray(b, np.float64)),
                                  pre, post, relax, smoother, _p(lab), m, coarse_tol, max_cycles, rel_tol, precision,
                                  _p(hist), {"V": 0, "W": 1}[cycle])
        return x, hist[: cyc + 1]


# ---------------------------------------------------------------------------
# Reference kernels compiled from the reference tree (oracle/_ref), for pinning
# ---------------------------------------------------------------------------
_ref = None


def set_threads(n):
    """Number of OpenMP threads of the oracle's parallel loops; returns the count in effect."""
    return int(lib().orc_set_threads(int(n)))


def divkgrad_element_matrix(X, kind=0, k4=None):
    """The oracle's restatement of p1_div_k_grad_affine_q3::integrateAll on the tetrahedron X
    (4 x 3): kind 0 with the P1 interpolant of the nodal values k4, kind 1 with
    k(x) = tanh(2 (x - 1/2)) + 2."""
    a = np.zeros(16)
    k = np.ascontiguousarray(np.ones(4) if k4 is None else k4, np.float64)
    if lib().orc_divkgrad_element_matrix(_p(np.ascontiguousarray(X, np.float64)), int(kind), _p(k), _p(a)) != 0:
        raise ValueError("unknown coefficient kind")
    return a.reshape(4, 4)


def chebyshev_coefficients(order, lower, upper):
    out = np.zeros(order)
    lib().orc_chebyshev_coefficients(order, lower, upper, _p(out))
    return out


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


_ref_face = None


def ref_face_lib():
    """The reference's generated macro-face kernels (oracle/ref_face_abi.cpp), or None."""
    global _ref_face
    if _ref_face is None:
        if not os.path.exists(REF_FACE_LIB):
            return None
        R = ctypes.CDLL(REF_FACE_LIB)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        R.ref_face_apply.argtypes = [P, P, P, I, P, P, I]
        R.ref_face_sor.argtypes = [P, P, P, P, I, P, P, D, P, P, I]
        R.ref_cell_to_face.argtypes = [P, P, I, P]
        R.ref_face_to_cell.argtypes = [P, P, I, P]
        _ref_face = R
    return _ref_face


# ---------------------------------------------------------------------------
# Synthetic inputs: one definition, shared with bench.py (hyb_inputs.py), so the
# oracle and the GPU path are fed identical, layout-independent values.
# ---------------------------------------------------------------------------
import sys as _sys  # noqa: E402

_INPUTS = os.path.join(os.path.dirname(HERE), "hyteg-vara_b200", "python")
if _INPUTS not in _sys.path:
    _sys.path.insert(0, _INPUTS)
from hyb_inputs import grf_coefficient, mesh_cuboid, splitmix64, uniform_rhs  # noqa: E402,F401


def _closure_map(self, level, cell):
    N = 1 << level
    out = np.zeros((N + 1) * (N + 2) * (N + 3) // 6, np.int32)
    lib().orc_cell_closure_map(self.h, level, cell, _p(out))
    return out


Oracle.closure_map = _closure_map
