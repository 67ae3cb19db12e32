"""Python binding of the B200 P1 multigrid C ABI (include/hyteg_b200.h).

Thin ctypes layer over hyteg-vara_b200/libhyteg_b200.so. Class and method names
follow the reference's C++ API (P1Function, P1ConstantLaplaceOperator,
P1ElementwiseDivKGradOperator, P1toP1LinearProlongation/Restriction, CGSolver,
GeometricMultigridSolver). There is no CPU fallback: if the shared library is
missing or no CUDA device is present, constructing any object raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libhyteg_b200.so")

INNER, DIRICHLET, NEUMANN, FREESLIP, ALL = 1, 2, 4, 8, 15
REPLACE, ADD = 0, 1
F64, F32 = 0, 1
SMOOTHER_SOR, SMOOTHER_JACOBI, SMOOTHER_SYMMETRIC_SOR, SMOOTHER_CHEBYSHEV = 0, 1, 2, 3
# SORSmoother / SymmetricSORSmoother in the reference's own sweep order
SMOOTHER_SOR_REFERENCE_ORDER, SMOOTHER_SYMMETRIC_SOR_REFERENCE_ORDER = 4, 5
CYCLE_V, CYCLE_W = 0, 1

# the C ABI symbols (include/hyteg_b200.h); tests check that the library exports all of them
SYMBOLS = [
    "hyb_last_error", "hyb_kernel_launch_count", "hyb_storage_create", "hyb_storage_create_cuboid", "hyb_storage_destroy", "hyb_storage_counts",
    "hyb_storage_num_dofs", "hyb_storage_mesh", "hyb_storage_dof_coords", "hyb_storage_colouring", "hyb_function_create",
    "hyb_function_destroy", "hyb_function_upload", "hyb_function_download", "hyb_function_upload_device",
    "hyb_function_download_device", "hyb_function_interpolate_const", "hyb_function_assign", "hyb_function_add",
    "hyb_function_dot", "hyb_function_copy_convert", "hyb_operator_create_laplace", "hyb_operator_create_divkgrad",
    "hyb_operator_create_divkgrad_callback", "hyb_operator_destroy", "hyb_operator_apply", "hyb_operator_residual",
    "hyb_operator_smooth_sor", "hyb_operator_smooth_jac", "hyb_operator_cell_stencil", "hyb_prolongate",
    "hyb_restrict", "hyb_cg_solve", "hyb_gmg_create", "hyb_gmg_destroy", "hyb_gmg_solve",
    "hyb_gmg_solve_to_tolerance", "hyb_function_dot_noalloc", "hyb_function_fill_uniform_random",
    "hyb_operator_create_divkgrad_rff", "hyb_operator_create_divkgrad_quadrature",
    "hyb_operator_create_divkgrad_callback_quadrature", "hyb_operator_create_blend_divkgrad", "hyb_server_create", "hyb_server_destroy", "hyb_server_footprint",
    "hyb_server_submit", "hyb_server_run", "hyb_server_result", "hyb_server_stats", "hyb_server_batch_stats", "hyb_rff_features",
    "hyb_storage_create_spherical_shell", "hyb_gmg_solve_fmg", "hyb_storage_create_from_gmsh",
    "hyb_operator_smooth_sor_backwards", "hyb_operator_smooth_sor_reference_order", "hyb_gmg_set_cycle_type", "hyb_gmg_setup_chebyshev",
    "hyb_gmg_set_timing", "hyb_gmg_timing_json", "hyb_gmg_timing_reset",
    "hyb_chebyshev_coefficients", "hyb_operator_estimate_spectral_radius", "hyb_server_mesh_bytes",
]

COEFF_CONSTANT, COEFF_LOGNORMAL, COEFF_RADIAL = 0, 1, 2
MESH_CUBOID, MESH_SHELL = 0, 1


class Request(ctypes.Structure):
    """hyb_request: one Poisson solve on the unit cube split into nx x ny x nz macro-cubes, or
    on the spherical shell with ntan = nx, nrad = ny (mesh = MESH_SHELL)."""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("level", ctypes.c_int),
                ("coefficient", ctypes.c_int), ("precision", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("rel_tol", ctypes.c_double), ("max_cycles", ctypes.c_int), ("mesh", ctypes.c_int)]


class RequestResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("cycles", ctypes.c_int), ("rel_residual", ctypes.c_double),
                ("arrival_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double),
                ("footprint_bytes", ctypes.c_size_t)]

_lib = None
# double k(const double* xyz, void* ctx): a coefficient callback
KFUN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)


class HybError(RuntimeError):
    pass


def load(path=LIB_PATH):
    """Load the shared library and declare the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise HybError(f"{path} is missing: build it with `python __graft_entry__.py build`")
    L = ctypes.CDLL(path)
    P, I, I64, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
    PP = ctypes.POINTER(ctypes.c_void_p)
    sig = {
        "hyb_last_error": (ctypes.c_char_p, []),
        "hyb_kernel_launch_count": (ctypes.c_longlong, []),
        "hyb_storage_create": (I, [P, I64, P, I64, I, PP]),
        "hyb_storage_create_cuboid": (I, [I, I, I, P, P, I, PP]),
        "hyb_storage_destroy": (I, [P]),
        "hyb_storage_counts": (I, [P, P]),
        "hyb_storage_num_dofs": (I64, [P, I]),
        "hyb_storage_mesh": (I, [P, P, P]),
        "hyb_storage_colouring": (I, [P, P, P]),
        "hyb_storage_dof_coords": (I, [P, I, P]),
        "hyb_function_create": (I, [P, I, I, I, PP]),
        "hyb_function_destroy": (I, [P]),
        "hyb_function_upload": (I, [P, I, P, P]),
        "hyb_function_download": (I, [P, I, P, P]),
        "hyb_function_upload_device": (I, [P, I, P, P]),
        "hyb_function_download_device": (I, [P, I, P, P]),
        "hyb_function_interpolate_const": (I, [P, I, D, I, P]),
        "hyb_function_assign": (I, [P, I, I, P, P, I, P]),
        "hyb_function_add": (I, [P, I, I, P, P, I, P]),
        "hyb_function_dot": (I, [P, P, I, I, P, P]),
        "hyb_function_copy_convert": (I, [P, P, I, P]),
        "hyb_operator_create_laplace": (I, [P, I, I, PP]),
        "hyb_operator_create_divkgrad": (I, [P, I, I, P, PP]),
        "hyb_operator_create_divkgrad_callback": (I, [P, I, I, P, P, PP]),
        "hyb_operator_destroy": (I, [P]),
        "hyb_operator_apply": (I, [P, P, P, I, I, I, P]),
        "hyb_operator_residual": (I, [P, P, P, P, I, I, P]),
        "hyb_operator_smooth_sor": (I, [P, P, P, D, I, I, P]),
        "hyb_operator_smooth_jac": (I, [P, P, P, P, D, I, I, P]),
        "hyb_operator_cell_stencil": (I, [P, I, I, I, P]),
        "hyb_prolongate": (I, [P, I, I, I, P]),
        "hyb_restrict": (I, [P, I, I, P]),
        "hyb_cg_solve": (I, [P, P, P, I, D, I, P, P, P]),
        "hyb_gmg_create": (I, [P, P, I, I, I, I, D, I, D, I, PP]),
        "hyb_gmg_destroy": (I, [P]),
        "hyb_gmg_solve": (I, [P, P, P, I, P]),
        "hyb_gmg_solve_to_tolerance": (I, [P, P, P, I, D, I, I, P, P, P]),
        "hyb_function_dot_noalloc": (I, [P, P, I, I, P, P]),
        "hyb_function_fill_uniform_random": (I, [P, I, ctypes.c_uint64, D, P]),
        "hyb_operator_create_divkgrad_rff": (I, [P, I, I, P, P, I, D, D, PP]),
        "hyb_operator_create_divkgrad_quadrature": (I, [P, I, I, I, P, P, I, D, D, PP]),
        "hyb_operator_create_divkgrad_callback_quadrature": (I, [P, I, I, KFUN, P, PP]),
        "hyb_operator_create_blend_divkgrad": (I, [P, I, I, D, PP]),
        "hyb_storage_create_spherical_shell": (I, [I, I, D, D, I, PP]),
        "hyb_gmg_solve_fmg": (I, [P, P, P, I, I, P]),
        "hyb_storage_create_from_gmsh": (I, [ctypes.c_char_p, I, PP]),
        "hyb_operator_smooth_sor_backwards": (I, [P, P, P, D, I, I, P]),
        "hyb_operator_smooth_sor_reference_order": (I, [P, P, P, D, I, I, I, P]),
        "hyb_gmg_set_cycle_type": (I, [P, I]),
        "hyb_gmg_set_timing": (I, [P, I]),
        "hyb_gmg_timing_json": (I, [P, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
        "hyb_gmg_timing_reset": (I, [P]),
        "hyb_gmg_setup_chebyshev": (I, [P, I, D, D]),
        "hyb_chebyshev_coefficients": (I, [I, D, D, P]),
        "hyb_operator_estimate_spectral_radius": (I, [P, P, P, I, I, P]),
        "hyb_server_mesh_bytes": (I, [P, P]),
        "hyb_server_create": (I, [ctypes.c_size_t, I, I, PP]),
        "hyb_server_destroy": (I, [P]),
        "hyb_server_footprint": (I, [P, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_size_t)]),
        "hyb_server_submit": (I, [P, ctypes.POINTER(Request), D, P, ctypes.POINTER(I)]),
        "hyb_server_run": (I, [P, D]),
        "hyb_server_result": (I, [P, I, ctypes.POINTER(RequestResult)]),
        "hyb_server_stats": (I, [P, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(I), ctypes.POINTER(I)]),
        "hyb_server_batch_stats": (I, [P, ctypes.POINTER(I), ctypes.POINTER(I)]),
        "hyb_rff_features": (I, [ctypes.c_uint64, D, I, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def kernel_launch_count():
    return int(load().hyb_kernel_launch_count())


def _check(code):
    if code != 0:
        msg = load().hyb_last_error().decode()
        raise HybError(f"hyteg_b200 error {code}: {msg}")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _stream(stream):
    return ctypes.c_void_p(int(stream) if stream else 0)


class PrimitiveStorage:
    """Macro-mesh (vertices, tetrahedra) plus the level hierarchy, resident on the GPU."""

    def __init__(self, coords=None, tets=None, max_level=0, cuboid=None):
        L = load()
        h = ctypes.c_void_p()
        if cuboid is not None:
            nx, ny, nz, lo, hi = cuboid
            lo = np.asarray(lo, np.float64)
            hi = np.asarray(hi, np.float64)
            _check(L.hyb_storage_create_cuboid(nx, ny, nz, _p(lo), _p(hi), max_level, ctypes.byref(h)))
        else:
            c = np.ascontiguousarray(coords, np.float64)
            t = np.ascontiguousarray(tets, np.int64)
            _check(L.hyb_storage_create(_p(c), len(c), _p(t), len(t), max_level, ctypes.byref(h)))
        self.h = h
        self.max_level = max_level

    @classmethod
    def cuboid(cls, nx, ny, nz, max_level, lo=(0, 0, 0), hi=(1, 1, 1)):
        return cls(cuboid=(nx, ny, nz, lo, hi), max_level=max_level)

    @classmethod
    def from_gmsh(cls, path, max_level):
        """MeshInfo::fromGmshFile: a Gmsh 2.2 ASCII tetrahedral mesh."""
        st = cls.__new__(cls)
        h = ctypes.c_void_p()
        _check(load().hyb_storage_create_from_gmsh(os.fsencode(path), max_level, ctypes.byref(h)))
        st.h, st.max_level = h, max_level
        return st

    @classmethod
    def spherical_shell(cls, ntan, nrad, rmin, rmax, max_level):
        """MeshInfo::meshSphericalShell(ntan, nrad, rmin, rmax) (SHELLMESH_CLASSIC; ntan - 1 a power
        of two): the reference's vertices, cells and cell order."""
        st = cls.__new__(cls)
        h = ctypes.c_void_p()
        _check(load().hyb_storage_create_spherical_shell(ntan, nrad, float(rmin), float(rmax), max_level,
                                                         ctypes.byref(h)))
        st.h, st.max_level = h, max_level
        return st

    def close(self):
        if getattr(self, "h", None):
            try:
                load().hyb_storage_destroy(self.h)
            except Exception:  # interpreter shutdown: module globals already gone
                pass
            self.h = None

    def __del__(self):
        self.close()

    def counts(self):
        c = np.zeros(4, np.int64)
        _check(load().hyb_storage_counts(self.h, _p(c)))
        return c

    def num_dofs(self, level):
        return int(load().hyb_storage_num_dofs(self.h, level))

    def mesh(self):
        c = self.counts()
        coords = np.zeros((c[0], 3))
        tets = np.zeros((c[3], 4), np.int64)
        _check(load().hyb_storage_mesh(self.h, _p(coords), _p(tets)))
        return coords, tets

    def dof_coords(self, level):
        out = np.zeros((self.num_dofs(level), 3))
        _check(load().hyb_storage_dof_coords(self.h, level, _p(out)))
        return out

    def colouring(self):
        m = ctypes.c_int()
        lab = np.zeros(self.counts()[0], np.int32)
        _check(load().hyb_storage_colouring(self.h, ctypes.byref(m), _p(lab)))
        return m.value, lab


class P1Function:
    """P1Function<double|float>(name, storage, minLevel, maxLevel)."""

    def __init__(self, name, storage, min_level, max_level, dtype=F64):
        self.name, self.storage, self.dtype = name, storage, dtype
        self.min_level, self.max_level = min_level, max_level
        h = ctypes.c_void_p()
        _check(load().hyb_function_create(storage.h, min_level, max_level, dtype, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            try:
                load().hyb_function_destroy(self.h)
            except Exception:  # interpreter shutdown: module globals already gone
                pass
            self.h = None

    def __del__(self):
        self.close()

    @property
    def np_dtype(self):
        return np.float64 if self.dtype == F64 else np.float32

    def set(self, values, level, stream=None):
        v = np.ascontiguousarray(values, self.np_dtype)
        assert v.size == self.storage.num_dofs(level)
        _check(load().hyb_function_upload(self.h, level, _p(v), _stream(stream)))

    def get(self, level, stream=None):
        out = np.zeros(self.storage.num_dofs(level), self.np_dtype)
        _check(load().hyb_function_download(self.h, level, _p(out), _stream(stream)))
        return out

    def set_host_ptr(self, ptr, level, stream=None):
        """Upload from a raw host pointer (e.g. pinned memory) in the canonical DoF order."""
        _check(load().hyb_function_upload(self.h, level, ctypes.c_void_p(ptr), _stream(stream)))

    def get_host_ptr(self, ptr, level, stream=None):
        _check(load().hyb_function_download(self.h, level, ctypes.c_void_p(ptr), _stream(stream)))

    def set_device(self, ptr, level, stream=None):
        _check(load().hyb_function_upload_device(self.h, level, ctypes.c_void_p(ptr), _stream(stream)))

    def get_device(self, ptr, level, stream=None):
        _check(load().hyb_function_download_device(self.h, level, ctypes.c_void_p(ptr), _stream(stream)))

    def interpolate(self, value, level, flag=ALL, stream=None):
        _check(load().hyb_function_interpolate_const(self.h, level, float(value), flag, _stream(stream)))

    def fill_uniform_random(self, level, seed, lattice, stream=None):
        """Seeded U[-1,1) values from a hash of each DoF's lattice position (device side;
        equals hyb_inputs.uniform_rhs on the DoF coordinates)."""
        _check(load().hyb_function_fill_uniform_random(self.h, level, int(seed), float(lattice), _stream(stream)))

    def _lincomb(self, fn, scalars, funcs, level, flag, stream):
        n = len(funcs)
        sc = np.ascontiguousarray(scalars, np.float64)
        arr = (ctypes.c_void_p * max(n, 1))(*[f.h.value for f in funcs])
        _check(fn(self.h, level, n, _p(sc), ctypes.cast(arr, ctypes.c_void_p), flag, _stream(stream)))

    def assign(self, scalars, funcs, level, flag=ALL, stream=None):
        self._lincomb(load().hyb_function_assign, scalars, funcs, level, flag, stream)

    def add(self, scalars, funcs, level, flag=ALL, stream=None):
        self._lincomb(load().hyb_function_add, scalars, funcs, level, flag, stream)

    def dot_global(self, other, level, flag=ALL, stream=None):
        out = ctypes.c_double()
        _check(load().hyb_function_dot(self.h, other.h, level, flag, ctypes.byref(out), _stream(stream)))
        return out.value

    def copy_from(self, other, level, stream=None):
        _check(load().hyb_function_copy_convert(self.h, other.h, level, _stream(stream)))


class _Operator:
    def close(self):
        if getattr(self, "h", None):
            try:
                load().hyb_operator_destroy(self.h)
            except Exception:  # interpreter shutdown: module globals already gone
                pass
            self.h = None

    def __del__(self):
        self.close()

    def apply(self, src, dst, level, flag, update=REPLACE, stream=None):
        _check(load().hyb_operator_apply(self.h, src.h, dst.h, level, flag, update, _stream(stream)))

    def residual(self, x, b, r, level, flag, stream=None):
        _check(load().hyb_operator_residual(self.h, x.h, b.h, r.h, level, flag, _stream(stream)))

    def smooth_sor(self, dst, rhs, relax, level, flag, stream=None):
        _check(load().hyb_operator_smooth_sor(self.h, dst.h, rhs.h, float(relax), level, flag, _stream(stream)))

    def smooth_sor_backwards(self, dst, rhs, relax, level, flag, stream=None):
        _check(load().hyb_operator_smooth_sor_backwards(self.h, dst.h, rhs.h, float(relax), level, flag,
                                                        _stream(stream)))

    def smooth_sor_reference_order(self, dst, rhs, relax, level, flag, backwards=False, stream=None):
        """One SOR sweep in the reference's V -> E -> F -> C lexicographic order
        (smooth_sor / smooth_sor_backwards, P1Operator.hpp:352-431)."""
        _check(load().hyb_operator_smooth_sor_reference_order(self.h, dst.h, rhs.h, float(relax), level, flag,
                                                              int(bool(backwards)), _stream(stream)))

    def smooth_gs(self, dst, rhs, level, flag, stream=None):
        self.smooth_sor(dst, rhs, 1.0, level, flag, stream)

    def smooth_gs_backwards(self, dst, rhs, level, flag, stream=None):
        self.smooth_sor_backwards(dst, rhs, 1.0, level, flag, stream)

    def estimate_spectral_radius(self, x, tmp, level, iterations):
        """chebyshev::estimateRadius: power iteration on D^-1 A (x is the start vector)."""
        r = ctypes.c_double()
        _check(load().hyb_operator_estimate_spectral_radius(self.h, x.h, tmp.h, level, iterations, ctypes.byref(r)))
        return r.value

    def smooth_jac(self, dst, rhs, src, relax, level, flag, stream=None):
        _check(load().hyb_operator_smooth_jac(self.h, dst.h, rhs.h, src.h, float(relax), level, flag,
                                              _stream(stream)))

    def cell_stencil(self, level, cell, mask=0):
        out = np.zeros(15)
        _check(load().hyb_operator_cell_stencil(self.h, level, cell, mask, _p(out)))
        return out


class P1ConstantLaplaceOperator(_Operator):
    def __init__(self, storage, min_level, max_level):
        self.storage = storage
        h = ctypes.c_void_p()
        _check(load().hyb_operator_create_laplace(storage.h, min_level, max_level, ctypes.byref(h)))
        self.h = h


class P1ElementwiseDivKGradOperator(_Operator):
    """P1ElementwiseOperator<p1_div_k_grad_affine_q3>; the coefficient is given by its nodal
    values on every level (canonical DoF order), i.e. its P1 interpolant."""

    def __init__(self, storage, min_level, max_level, nodal_k):
        self.storage = storage
        arrs = [np.ascontiguousarray(k, np.float64) for k in nodal_k]
        ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        h = ctypes.c_void_p()
        _check(load().hyb_operator_create_divkgrad(storage.h, min_level, max_level, ctypes.cast(ptrs, ctypes.c_void_p),
                                                   ctypes.byref(h)))
        self.h = h

    @classmethod
    def random_features(cls, storage, min_level, max_level, w, phase, sigma, radial=0.0):
        """k(x) = exp(radial (1 - |x|) + sigma sqrt(2/M) sum_m cos(w_m . x + phase_m)),
        evaluated on the device."""
        w = np.ascontiguousarray(w, np.float64).reshape(-1, 3)
        phase = np.ascontiguousarray(phase, np.float64).ravel()
        assert w.shape[0] == phase.shape[0]
        op = cls.__new__(cls)
        op.storage = storage
        h = ctypes.c_void_p()
        _check(load().hyb_operator_create_divkgrad_rff(storage.h, min_level, max_level, w.ctypes.data,
                                                       phase.ctypes.data, w.shape[0], float(sigma), float(radial),
                                                       ctypes.byref(h)))
        op.h = h
        return op

    @classmethod
    def callback_quadrature(cls, storage, min_level, max_level, k):
        """Any coefficient k(xyz) -> float, called on the host at the 5 quadrature points of
        every micro-tet on every level (the reference form's callback semantics)."""
        op = cls.__new__(cls)
        op.storage = storage
        op._kfun = KFUN(lambda xyz, ctx: float(k(np.ctypeslib.as_array(xyz, shape=(3,)))))
        h = ctypes.c_void_p()
        _check(load().hyb_operator_create_divkgrad_callback_quadrature(storage.h, min_level, max_level, op._kfun,
                                                                       None, ctypes.byref(h)))
        op.h = h
        return op

    @classmethod
    def quadrature(cls, storage, min_level, max_level, kind, w=None, phase=None, sigma=1.0, radial=0.0):
        """The coefficient callback evaluated as the reference's form does: k at the 5
        quadrature points of every micro-tet on every level. kind 1: tanh(2 (x - 1/2)) + 2;
        kind 2: the random-feature field of random_features (w, phase, sigma, radial)."""
        op = cls.__new__(cls)
        op.storage = storage
        h = ctypes.c_void_p()
        if kind == 2:
            w = np.ascontiguousarray(w, np.float64).reshape(-1, 3)
            phase = np.ascontiguousarray(phase, np.float64).ravel()
            assert w.shape[0] == phase.shape[0]
            wp, pp, m = w.ctypes.data, phase.ctypes.data, w.shape[0]
        else:
            wp, pp, m = None, None, 0
        _check(load().hyb_operator_create_divkgrad_quadrature(storage.h, min_level, max_level, kind, wp, pp, m,
                                                              float(sigma), float(radial), ctypes.byref(h)))
        op.h = h
        return op


class P1ElementwiseBlendingDivKGradOperator(_Operator):
    """P1ElementwiseOperator<p1_div_k_grad_blending_q3> on a spherical-shell mesh whose cells
    carry the IcosahedralShellMap (IcosahedralShellMap::setMap); the coefficient is
    k(y) = exp(alpha (1 - |y|)) at the mapped quadrature points (alpha = 0: Laplacian).
    Element matrices are integrated on the device per row; levels up to 7."""

    def __init__(self, storage, min_level, max_level, alpha=0.0):
        self.storage = storage
        h = ctypes.c_void_p()
        _check(load().hyb_operator_create_blend_divkgrad(storage.h, min_level, max_level, float(alpha),
                                                         ctypes.byref(h)))
        self.h = h


class P1toP1LinearProlongation:
    def prolongate(self, f, source_level, flag, stream=None):
        _check(load().hyb_prolongate(f.h, source_level, flag, REPLACE, _stream(stream)))

    def prolongate_and_add(self, f, source_level, flag, stream=None):
        _check(load().hyb_prolongate(f.h, source_level, flag, ADD, _stream(stream)))


class P1toP1LinearRestriction:
    def restrict(self, f, source_level, flag, stream=None):
        _check(load().hyb_restrict(f.h, source_level, flag, _stream(stream)))


class CGSolver:
    def __init__(self, tolerance=1e-16, max_iter=100000):
        self.tolerance, self.max_iter = tolerance, max_iter

    def solve(self, A, x, b, level, stream=None):
        it, conv = ctypes.c_int(), ctypes.c_int()
        _check(load().hyb_cg_solve(A.h, x.h, b.h, level, self.tolerance, self.max_iter, ctypes.byref(it),
                                   ctypes.byref(conv), _stream(stream)))
        return it.value, conv.value == 1


class GeometricMultigridSolver:
    """GeometricMultigridSolver(storage, smoother, coarseSolver, restriction, prolongation,
    minLevel, maxLevel, preSmooth, postSmooth): solve() performs one V-cycle."""

    def __init__(self, storage, A, min_level, max_level, pre=3, post=3, relax=1.0, smoother=SMOOTHER_SOR,
                 coarse_tol=1e-12, coarse_max_iter=10000, cycle_type=CYCLE_V):
        self.storage, self.A = storage, A
        h = ctypes.c_void_p()
        _check(load().hyb_gmg_create(storage.h, A.h, min_level, max_level, pre, post, float(relax), smoother,
                                     float(coarse_tol), coarse_max_iter, ctypes.byref(h)))
        self.h = h
        if cycle_type != CYCLE_V:
            _check(load().hyb_gmg_set_cycle_type(self.h, cycle_type))

    def setup_chebyshev(self, order, spectral_radius=None, lower=None, upper=None):
        """ChebyshevSmoother::setupCoefficients(order, rho) -> [0.3 rho, 1.2 rho], or explicit
        bounds of the eigenvalue interval of D^-1 A."""
        if spectral_radius is not None:
            lower, upper = 0.3 * spectral_radius, 1.2 * spectral_radius
        _check(load().hyb_gmg_setup_chebyshev(self.h, order, float(lower), float(upper)))

    def close(self):
        if getattr(self, "h", None):
            try:
                load().hyb_gmg_destroy(self.h)
            except Exception:  # interpreter shutdown: module globals already gone
                pass
            self.h = None

    def __del__(self):
        self.close()

    def solve(self, x, b, level, stream=None):
        _check(load().hyb_gmg_solve(self.h, x.h, b.h, level, _stream(stream)))

    def set_timing(self, enable=True):
        """Stage timers in the reference's timing-tree shape (device events); while on, solves
        run launch by launch."""
        _check(load().hyb_gmg_set_timing(self.h, int(bool(enable))))

    def timing(self):
        """The accumulated timing tree: {name: {total, average, min, max, count, children}}."""
        import json

        n = ctypes.c_size_t()
        _check(load().hyb_gmg_timing_json(self.h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        _check(load().hyb_gmg_timing_json(self.h, buf, n.value + 1, ctypes.byref(n)))
        return json.loads(buf.value.decode())

    def reset_timing(self):
        _check(load().hyb_gmg_timing_reset(self.h))

    def solve_fmg(self, x, b, level, cycles_per_level=1, stream=None):
        """FullMultigridSolver::solve: b must hold the right-hand side on every level."""
        _check(load().hyb_gmg_solve_fmg(self.h, x.h, b.h, level, cycles_per_level, _stream(stream)))

    def solve_to_tolerance(self, x, b, level, rel_tol, max_cycles=100, precision=64, stream=None):
        hist = np.zeros(max_cycles + 1)
        cyc = ctypes.c_int()
        _check(load().hyb_gmg_solve_to_tolerance(self.h, x.h, b.h, level, float(rel_tol), max_cycles, precision,
                                                 _p(hist), ctypes.byref(cyc), _stream(stream)))
        return hist[: cyc.value + 1]


def chebyshev_coefficients(order, lower, upper):
    out = np.zeros(order)
    _check(load().hyb_chebyshev_coefficients(order, float(lower), float(upper), _p(out)))
    return out


def rff_features(seed, corr_len=0.2, modes=64):
    """The random Fourier features the server draws for a lognormal request of this seed."""
    w, ph = np.zeros((modes, 3)), np.zeros(modes)
    _check(load().hyb_rff_features(int(seed), float(corr_len), modes, w.ctypes.data, ph.ctypes.data))
    return w, ph


class Server:
    """Continuous-batching serving loop (hyb_server_*): submit requests with arrival times,
    run, read per-request results."""

    def __init__(self, budget_bytes, max_active=16, max_level=7):
        h = ctypes.c_void_p()
        _check(load().hyb_server_create(int(budget_bytes), max_active, max_level, ctypes.byref(h)))
        self.h = h
        self._solutions = {}

    def close(self):
        if getattr(self, "h", None):
            try:
                load().hyb_server_destroy(self.h)
            except Exception:  # interpreter shutdown: module globals already gone
                pass
            self.h = None

    def __del__(self):
        self.close()

    @staticmethod
    def request(nx, ny, nz, level, coefficient=COEFF_CONSTANT, precision=32, seed=0, rel_tol=1e-8, max_cycles=100,
                mesh=MESH_CUBOID):
        return Request(nx, ny, nz, level, coefficient, precision, seed, rel_tol, max_cycles, mesh)

    def footprint(self, req):
        n = ctypes.c_size_t()
        _check(load().hyb_server_footprint(self.h, ctypes.byref(req), ctypes.byref(n)))
        return n.value

    def submit(self, req, arrival_s=0.0, keep_solution=False, num_dofs=None):
        """Returns the request id. keep_solution needs num_dofs (hyb_storage_num_dofs of the
        request's mesh and level)."""
        buf = None
        if keep_solution:
            buf = np.zeros(int(num_dofs))
        i = ctypes.c_int()
        _check(load().hyb_server_submit(self.h, ctypes.byref(req), float(arrival_s),
                                        buf.ctypes.data if buf is not None else None, ctypes.byref(i)))
        if buf is not None:
            self._solutions[i.value] = buf
        return i.value

    def run(self, time_limit_s=600.0):
        _check(load().hyb_server_run(self.h, float(time_limit_s)))

    def result(self, rid):
        r = RequestResult()
        _check(load().hyb_server_result(self.h, rid, ctypes.byref(r)))
        return r

    def solution(self, rid):
        return self._solutions[rid]

    def stats(self):
        peak, built, graphs = ctypes.c_size_t(), ctypes.c_int(), ctypes.c_int()
        _check(load().hyb_server_stats(self.h, ctypes.byref(peak), ctypes.byref(built), ctypes.byref(graphs)))
        mesh = ctypes.c_size_t()
        _check(load().hyb_server_mesh_bytes(self.h, ctypes.byref(mesh)))
        batches, batched = ctypes.c_int(), ctypes.c_int()
        _check(load().hyb_server_batch_stats(self.h, ctypes.byref(batches), ctypes.byref(batched)))
        return {"peak_bytes": peak.value, "hierarchies_built": built.value, "graphs_captured": graphs.value,
                "mesh_bytes": mesh.value, "batches": batches.value, "batched_solves": batched.value}
