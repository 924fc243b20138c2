"""B200-native BK/BP Hex3D hot path: Python binding of libbp_b200.so.

The library (include/bp_b200.h) replaces benchParanumal's OCCA platform layer
and OKL kernels for the Hex3D BK/BP path.  This module mirrors the reference's
host objects for that path:

    Mesh      mesh_t for the Hex3D box + its masked ogs numbering
              (libs/mesh/meshSetup.cpp, meshMaskedGatherScatterSetup.cpp)
    BP        bpN_t : solver_t with Operator / forcing / cg::Solve
              (BP/BP5/src/bp5{Setup,Operator,Run}.cpp, libs/core/linearSolverCG.cpp)
    ax_hex3d  the bp5AxHex3D / bp5AxAffineHex3D / bp6AxHex3D kernels
    ax_cub_hex3d  the over-integrated bp1-bp4 (Affine) Hex3D kernels
    ogs_gather / ogs_scatter   the ogs Gather(Add, Trans) / Scatter(NoTrans)

Errors raise BPError carrying the library's message, the way the reference
throws libp::exception.  There is no CPU fallback: without the built library
or without a CUDA device every call fails loudly.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libbp_b200.so")

BP_SUCCESS = 0
BP_ERROR = -1
BP_ERROR_ARG = -2
BP_ERROR_CUDA = -3
BP_ERROR_ALLOC = -4
BP_ERROR_NUMERIC = -5
BP_ERROR_TIMEOUT = -6
BP_PRECON_NONE = 0
BP_PRECON_JACOBI = 1
BP_RHS_ANALYTIC = 0
BP_RHS_RANDOM = 1
BP_PRECISION_FP64 = 0
BP_PRECISION_MIXED = 1

EXPORTS = [
    "bp_last_error", "bp_version", "bp_platform_init", "bp_device_count", "bp_device_info",
    "bp_malloc", "bp_free", "bp_host_malloc", "bp_host_free", "bp_memcpy_htod", "bp_memcpy_dtoh",
    "bp_memcpy_dtod", "bp_memset", "bp_stream_create", "bp_stream_destroy", "bp_finish",
    "bp_event_create", "bp_event_destroy", "bp_event_record", "bp_event_elapsed_ms",
    "bp_ax_hex3d", "bp_ax_tri2d", "bp_ax_tet3d", "bp_ogs_gather", "bp_ogs_scatter", "bp_linalg_set", "bp_linalg_axpy",
    "bp_linalg_inner_prod", "bp_linalg_norm2", "bp_update_cg",
    "bp_mesh_create", "bp_mesh_view", "bp_mesh_destroy",
    "bp_solver_create", "bp_solver_destroy", "bp_solver_size", "bp_solver_operator", "bp_solver_rhs",
    "bp_solver_diagonal", "bp_solver_solve", "bp_solver_solve_host", "bp_driver_main",
    "bp_box_numbering", "bp_basis_gll", "bp_box_vertices", "bp_operator_hex3d_noalloc", "bp_ogs_check",
    "bp_test_wait_timeout", "bp_tune_report", "bp_tune_reset",
    "bp_ax_cub_hex3d", "bp_mesh_cubature", "bp_mesh_cubature_view", "bp_basis_cubature", "bp_basis_tri2d", "bp_basis_tet3d",
    "bp_batch_create", "bp_batch_destroy", "bp_batch_systems", "bp_batch_system_info", "bp_batch_solve",
    "bp_batch_vectors", "bp_batch_solver", "bp_ax_hex3d_f32", "bp_convert_f64_f32", "bp_ax_hex3d_f32_multi",
    "bp_ax_cub_hex3d_f32", "bp_mesh_write_vtu", "bp_ogs_owner_map", "bp_cg_direction_ax_hex3d",
    "bp_cg_direction_ax_f32_multi",
]


class BPError(RuntimeError):
    """A C-ABI call returned an error status (libp::exception equivalent)."""

    def __init__(self, code, msg):
        super().__init__("bp error %d: %s" % (code, msg))
        self.code = code


class AxDesc(ctypes.Structure):
    _fields_ = [("bp", ctypes.c_int32), ("N", ctypes.c_int32), ("affine", ctypes.c_int32),
                ("Nfields", ctypes.c_int32), ("dim", ctypes.c_int32)]


class BoxDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("N", ctypes.c_int32),
                ("affine", ctypes.c_int32), ("Nfields", ctypes.c_int32), ("pert", ctypes.c_double),
                ("pert_seed", ctypes.c_uint64), ("dim", ctypes.c_int32), ("simplex", ctypes.c_int32)]


class MeshView(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int32), ("Nq", ctypes.c_int32), ("Np", ctypes.c_int32),
                ("Nelements", ctypes.c_int32), ("Nfields", ctypes.c_int32), ("affine", ctypes.c_int32),
                ("Ngather", ctypes.c_int32), ("nnz", ctypes.c_int32), ("Nlocal", ctypes.c_int64)] + [
        (n, ctypes.c_void_p) for n in ("elementList", "GlobalToLocal", "rowStarts", "colIds", "wJ", "ggeo", "D",
                                       "gllz", "gllw", "EX", "EY", "EZ")] + [("dim", ctypes.c_int32),
                                                                              ("simplex", ctypes.c_int32),
                                                                              ("S", ctypes.c_void_p),
                                                                              ("MM", ctypes.c_void_p)]


def _ax_desc(mesh, bp=None):
    """The operator descriptor of a mesh: BP5 with one field, BP6 with more."""
    if bp is None:
        bp = 6 if mesh.Nfields > 1 else 5
    nf = 1 if bp == 5 else mesh.Nfields
    return AxDesc(bp, mesh.N, int(mesh.affine), nf, getattr(mesh, "dim", 3))


class CubatureView(ctypes.Structure):
    _fields_ = [("cubNq", ctypes.c_int32), ("cubNp", ctypes.c_int32)] + [
        (n, ctypes.c_void_p) for n in ("cubr", "cubw", "cubInterp", "cubD", "invV", "MM", "cubwJ", "cubggeo")]


class BatchProblem(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("N", ctypes.c_int32),
                ("pert", ctypes.c_double), ("pert_seed", ctypes.c_uint64), ("nrhs", ctypes.c_int32),
                ("rhs_seed", ctypes.c_uint64), ("affine", ctypes.c_int32)]


class SolverDesc(ctypes.Structure):
    _fields_ = [("bp", ctypes.c_int32), ("lambda_", ctypes.c_double), ("precon", ctypes.c_int32),
                ("precision", ctypes.c_int32)]


class SolveStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("rdotr0", ctypes.c_double), ("rdotr", ctypes.c_double),
                ("elapsed_ms", ctypes.c_double), ("updates", ctypes.c_int32), ("kernel_launches", ctypes.c_int64)]


_lib = None


def lib():
    """Load libbp_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BPError(-1, "libbp_b200.so is not built; run python -m benchparanumal_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, dbl, u64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_uint64
        sz = ctypes.c_size_t
        L.bp_last_error.restype = ctypes.c_char_p
        L.bp_version.restype = ctypes.c_char_p
        sigs = {
            "bp_platform_init": [ctypes.c_int],
            "bp_device_count": [ctypes.POINTER(ctypes.c_int)],
            "bp_device_info": [ctypes.c_char_p, sz, ctypes.POINTER(ctypes.c_int)],
            "bp_malloc": [ctypes.POINTER(vp), sz],
            "bp_free": [vp],
            "bp_host_malloc": [ctypes.POINTER(vp), sz],
            "bp_host_free": [vp],
            "bp_memcpy_htod": [vp, vp, sz, vp],
            "bp_memcpy_dtoh": [vp, vp, sz, vp],
            "bp_memcpy_dtod": [vp, vp, sz, vp],
            "bp_memset": [vp, ctypes.c_int, sz, vp],
            "bp_stream_create": [ctypes.POINTER(vp)],
            "bp_stream_destroy": [vp],
            "bp_finish": [vp],
            "bp_event_create": [ctypes.POINTER(vp)],
            "bp_event_destroy": [vp],
            "bp_event_record": [vp, vp],
            "bp_event_elapsed_ms": [vp, vp, ctypes.POINTER(ctypes.c_float)],
            "bp_ax_hex3d": [ctypes.POINTER(AxDesc), i32, vp, vp, vp, vp, vp, vp, dbl, vp, vp, vp],
            "bp_ax_tri2d": [ctypes.POINTER(AxDesc), i32, vp, vp, vp, vp, vp, vp, dbl, vp, vp, vp],
            "bp_ax_tet3d": [ctypes.POINTER(AxDesc), i32, vp, vp, vp, vp, vp, vp, dbl, vp, vp, vp],
            "bp_ogs_gather": [i32, vp, vp, vp, vp, vp],
            "bp_ogs_scatter": [i32, vp, vp, vp, vp, vp],
            "bp_linalg_set": [i32, dbl, vp, vp],
            "bp_linalg_axpy": [i32, dbl, vp, dbl, vp, vp],
            "bp_linalg_inner_prod": [i32, vp, vp, vp, vp],
            "bp_linalg_norm2": [i32, vp, vp, vp],
            "bp_update_cg": [i32, vp, dbl, vp, vp, vp],
            "bp_mesh_create": [ctypes.POINTER(BoxDesc), ctypes.POINTER(vp)],
            "bp_mesh_view": [vp, ctypes.POINTER(MeshView)],
            "bp_mesh_destroy": [vp],
            "bp_solver_create": [vp, ctypes.POINTER(SolverDesc), ctypes.POINTER(vp)],
            "bp_solver_destroy": [vp],
            "bp_solver_size": [vp, ctypes.POINTER(i32)],
            "bp_solver_operator": [vp, vp, vp, vp],
            "bp_solver_rhs": [vp, i32, u64, vp, vp],
            "bp_solver_diagonal": [vp, vp],
            "bp_solver_solve": [vp, vp, vp, dbl, i32, vp, vp, ctypes.POINTER(SolveStats)],
            "bp_solver_solve_host": [vp, vp, vp, dbl, i32, ctypes.POINTER(SolveStats)],
            "bp_driver_main": [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)],
            "bp_box_numbering": [ctypes.POINTER(BoxDesc), ctypes.POINTER(i32), ctypes.POINTER(i32), vp, vp, vp],
            "bp_basis_gll": [i32, vp, vp, vp],
            "bp_box_vertices": [ctypes.POINTER(BoxDesc), vp, vp, vp],
            "bp_ogs_check": [ctypes.c_int64, vp, i32, vp, vp],
            "bp_test_wait_timeout": [ctypes.c_int],
            "bp_tune_report": [i32] * 8 + [ctypes.POINTER(i32), ctypes.POINTER(i32), vp, vp, i32],
            "bp_tune_reset": [],
            "bp_operator_hex3d_noalloc": [ctypes.POINTER(AxDesc), i32, vp, vp, vp, vp, vp, vp, dbl, i32, i32, vp,
                                          vp, vp, vp, vp],
            "bp_ax_cub_hex3d": [ctypes.POINTER(AxDesc), i32, vp, vp, vp, vp, vp, vp, vp, vp, dbl, vp, vp, vp],
            "bp_mesh_cubature": [vp],
            "bp_basis_tri2d": [i32, vp, vp, vp, vp, vp],
            "bp_basis_tet3d": [i32, vp, vp, vp, vp, vp, vp],
            "bp_mesh_cubature_view": [vp, ctypes.POINTER(CubatureView)],
            "bp_basis_cubature": [i32, vp, vp, vp, vp, vp, vp, vp],
            "bp_batch_create": [ctypes.POINTER(BatchProblem), i32, ctypes.POINTER(SolverDesc), ctypes.POINTER(vp)],
            "bp_batch_destroy": [vp],
            "bp_batch_systems": [vp, ctypes.POINTER(i32)],
            "bp_batch_system_info": [vp, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)],
            "bp_batch_solve": [vp, dbl, i32, ctypes.POINTER(SolveStats), ctypes.POINTER(dbl)],
            "bp_batch_vectors": [vp, i32, ctypes.POINTER(vp), ctypes.POINTER(vp)],
            "bp_batch_solver": [vp, i32, ctypes.POINTER(vp)],
            "bp_ax_hex3d_f32": [ctypes.POINTER(AxDesc), i32, vp, vp, vp, vp, vp, vp, ctypes.c_float, vp, vp, vp],
            "bp_convert_f64_f32": [sz, vp, vp, vp],
            "bp_ax_hex3d_f32_multi": [ctypes.POINTER(AxDesc), i32, i32, vp, vp, vp, vp, vp, vp, ctypes.c_float, vp, vp,
                                      vp],
            "bp_ax_cub_hex3d_f32": [ctypes.POINTER(AxDesc), i32, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_float, vp, vp,
                                    vp],
            "bp_mesh_write_vtu": [vp, vp, ctypes.c_char_p],
            "bp_ogs_owner_map": [i32, vp, i32, vp, vp, vp, vp],
            "bp_cg_direction_ax_hex3d": [ctypes.POINTER(AxDesc), i32, vp, vp, vp, vp, vp, dbl, dbl, dbl, vp, vp, vp,
                                         vp, vp, vp, vp, vp],
            "bp_cg_direction_ax_f32_multi": [ctypes.POINTER(AxDesc), i32, i32, vp, vp, vp, vp, vp, ctypes.c_float,
                                             vp, vp, vp, vp, vp, vp, vp, vp, vp, vp],
        }
        for name, args in sigs.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def _check(rc):
    if rc != BP_SUCCESS:
        raise BPError(rc, lib().bp_last_error().decode(errors="replace"))


_initialised = None


def platform_init(device=0):
    """-m CUDA -d <device>: select the device (sm_100a required)."""
    global _initialised
    if _initialised != device:
        _check(lib().bp_platform_init(device))
        _initialised = device


def finish():
    """platform.finish(): wait for the library's stream."""
    _check(lib().bp_finish(None))


class DeviceBuffer:
    """A device allocation from bp_malloc holding `n` items of `dtype`."""

    def __init__(self, n, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        self.n = int(n)
        self.nbytes = self.n * self.dtype.itemsize
        p = ctypes.c_void_p()
        _check(lib().bp_malloc(ctypes.byref(p), self.nbytes))
        self.ptr = p.value or 0

    @classmethod
    def from_host(cls, a):
        a = np.ascontiguousarray(a)
        b = cls(a.size, a.dtype)
        b.upload(a)
        return b

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        assert a.size == self.n
        _check(lib().bp_memcpy_htod(self.ptr, a.ctypes.data, self.nbytes, None))
        finish()

    def download(self):
        out = np.empty(self.n, dtype=self.dtype)
        _check(lib().bp_memcpy_dtoh(out.ctypes.data, self.ptr, self.nbytes, None))
        finish()
        return out

    def zero(self):
        _check(lib().bp_memset(self.ptr, 0, self.nbytes, None))

    def free(self):
        if getattr(self, "ptr", 0):
            lib().bp_free(self.ptr)
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PinnedBuffer:
    """Page-locked host memory from bp_host_malloc, viewed as a numpy array."""

    def __init__(self, n, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        self.n = int(n)
        p = ctypes.c_void_p()
        _check(lib().bp_host_malloc(ctypes.byref(p), self.n * self.dtype.itemsize))
        self.ptr = p.value or 0
        ct = np.ctypeslib.as_ctypes_type(self.dtype)
        self.array = np.frombuffer((ct * self.n).from_address(self.ptr), dtype=self.dtype) if self.n else \
            np.empty(0, self.dtype)

    def free(self):
        if getattr(self, "ptr", 0):
            self.array = None
            lib().bp_host_free(self.ptr)
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _dl(ptr, n, dtype):
    out = np.empty(n, dtype=dtype)
    if n:
        _check(lib().bp_memcpy_dtoh(out.ctypes.data, ptr, out.nbytes, None))
        finish()
    return out


class Mesh:
    """Box mesh on the device (mesh_t + masked ogs), built by bp_mesh_create:
    Hex3D, or Quad2D with dim=2 (nz ignored; Nfields 1 or 2), or Tri2D with
    dim=2 and simplex=True (affine, one field, 2*nx*ny triangles), or Tet3D with
    dim=3 and simplex=True (6*nx*ny*nz tetrahedra)."""

    def __init__(self, nx, ny=None, nz=None, N=4, affine=False, Nfields=1, pert=0.0, pert_seed=1, device=0, dim=3,
                 simplex=False):
        platform_init(device)
        ny = nx if ny is None else ny
        nz = (nx if nz is None else nz) if dim == 3 else 1
        d = BoxDesc(nx, ny, nz, N, int(bool(affine)), Nfields, float(pert), int(pert_seed), int(dim),
                    int(bool(simplex)))
        h = ctypes.c_void_p()
        _check(lib().bp_mesh_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h.value
        self.view = MeshView()
        _check(lib().bp_mesh_view(self._h, ctypes.byref(self.view)))
        v = self.view
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dim = v.dim
        self.simplex = bool(v.simplex)
        self.N, self.Nq, self.Np, self.E = v.N, v.Nq, v.Np, v.Nelements
        self.Nfields, self.affine = v.Nfields, bool(v.affine)
        self.Ngather, self.nnz, self.NL = v.Ngather, v.nnz, int(v.Nlocal)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().bp_mesh_destroy(self._h)
            self._h = None

    def array(self, name):
        """Copy a device mesh array to the host (names as in bp_mesh_view_t)."""
        v = self.view
        ng = self.E if self.affine else self.E * self.Np
        if self.simplex:
            nv, ngg = (3, 3) if self.dim == 2 else (4, 6)
        else:
            nv, ngg = (8, 6) if self.dim == 3 else (4, 3)
        if self.simplex:   # D holds Dr, Ds (, Dt), S the stiffness matrices, MM the mass matrix
            NP2 = self.Np * self.Np
            tri = {"D": self.dim * NP2, "S": (3 if self.dim == 2 else 6) * NP2, "MM": NP2}
            if name in tri:
                return _dl(getattr(v, name), tri[name], np.float64)
        spec = {
            "elementList": (self.E, np.int32), "GlobalToLocal": (self.NL, np.int32),
            "rowStarts": (self.Ngather + 1, np.int32), "colIds": (self.nnz, np.int32),
            "wJ": (ng, np.float64), "ggeo": (ngg * ng, np.float64), "D": (self.Nq * self.Nq, np.float64),
            "gllz": (self.Nq, np.float64), "gllw": (self.Nq, np.float64), "EX": (nv * self.E, np.float64),
            "EY": (nv * self.E, np.float64), "EZ": ((nv if self.dim == 3 else 0) * self.E, np.float64),
        }
        if name in spec:
            n, dt = spec[name]
            return _dl(getattr(v, name), n, dt)
        c = self.cubature()
        G, Nq = c.cubNq, self.Nq
        ncub = self.E if self.affine else self.E * c.cubNp
        cspec = {
            "cubr": G, "cubw": G, "cubInterp": G * Nq, "cubD": (Nq * Nq if self.affine else G * G),
            "invV": Nq * Nq, "MM": Nq * Nq, "cubwJ": ncub, "cubggeo": 6 * ncub,
        }
        return _dl(getattr(c, name), cspec[name], np.float64)

    def write_vtu(self, xL, filename):
        """bp_mesh_write_vtu: write a host E-vector [E*Np*Nfields] as a VTK XML grid."""
        a = np.ascontiguousarray(xL, dtype=np.float64)
        if a.size != self.NL:
            raise ValueError("xL must hold E*Np*Nfields values")
        _check(lib().bp_mesh_write_vtu(self._h, a.ctypes.data, str(filename).encode()))

    def cubature(self):
        """Set up (once) and return the cubature view of the BP1-BP4 operators."""
        if getattr(self, "_cub", None) is None:
            _check(lib().bp_mesh_cubature(self._h))
            c = CubatureView()
            _check(lib().bp_mesh_cubature_view(self._h, ctypes.byref(c)))
            self._cub = c
        return self._cub


def ax_hex3d(mesh, q, Aq, lam=1.0, elementList=None, Nelements=None, stream=None):
    """bp_ax_hex3d on device buffers: Aq (E-vector) = A_e q[GlobalToLocal]."""
    v = mesh.view
    d = _ax_desc(mesh)
    el = v.elementList if elementList is None else elementList
    ne = mesh.E if Nelements is None else Nelements
    _check(lib().bp_ax_hex3d(ctypes.byref(d), ne, el, v.GlobalToLocal, v.wJ, v.ggeo, v.gllw, v.D, float(lam),
                             _ptr(q), _ptr(Aq), stream))


def ax_cub_hex3d(mesh, bp, q, Aq, lam=1.0, stream=None):
    """bp_ax_cub_hex3d on device buffers: the over-integrated BP1-BP4 element
    operator, Aq (E-vector) = A_e q[GlobalToLocal]."""
    v, c = mesh.view, mesh.cubature()
    d = AxDesc(bp, mesh.N, int(mesh.affine), mesh.Nfields)
    _check(lib().bp_ax_cub_hex3d(ctypes.byref(d), mesh.E, v.elementList, v.GlobalToLocal, c.cubwJ, c.cubggeo,
                                 c.cubD, c.cubInterp, c.invV, c.MM, float(lam), _ptr(q), _ptr(Aq), stream))


def convert_f64_f32(src, n, dst, stream=None):
    """dst (FP32 device) = src (FP64 device address or buffer), n elements."""
    _check(lib().bp_convert_f64_f32(n, src if isinstance(src, int) else _ptr(src), _ptr(dst), stream))


def ax_tet3d(mesh, q, Aq, lam=1.0, stream=None):
    """bp_ax_tet3d on a Tet3D mesh's own arrays: Aq (E-vector) = A_e q[G2L]."""
    v = mesh.view
    d = AxDesc(5, mesh.N, 1, 1, 3)
    _check(lib().bp_ax_tet3d(ctypes.byref(d), mesh.E, v.elementList, v.GlobalToLocal, v.wJ, v.ggeo, v.S, v.MM,
                             float(lam), q.ptr, Aq.ptr, stream))


def ax_tri2d(mesh, q, Aq, lam=1.0, stream=None):
    """bp_ax_tri2d on a Tri2D mesh's own arrays: Aq (E-vector) = A_e q[G2L]."""
    v = mesh.view
    d = AxDesc(5, mesh.N, 1, 1, 2)
    _check(lib().bp_ax_tri2d(ctypes.byref(d), mesh.E, v.elementList, v.GlobalToLocal, v.wJ, v.ggeo, v.S, v.MM,
                             float(lam), q.ptr, Aq.ptr, stream))


def ax_hex3d_f32(mesh, q, Aq, ops, lam=1.0, stream=None):
    """bp_ax_hex3d_f32 on FP32 device buffers; ops = dict of FP32 buffers wJ, ggeo, gllw, D."""
    v = mesh.view
    d = _ax_desc(mesh)
    _check(lib().bp_ax_hex3d_f32(ctypes.byref(d), mesh.E, v.elementList, v.GlobalToLocal, _ptr(ops["wJ"]),
                                 _ptr(ops["ggeo"]), _ptr(ops["gllw"]), _ptr(ops["D"]), float(lam), _ptr(q),
                                 _ptr(Aq), stream))


def ax_hex3d_f32_multi(mesh, nrhs, q, Aq, ops, lam=1.0, stream=None):
    """bp_ax_hex3d_f32_multi: the FP32 operator on nrhs interleaved right-hand sides."""
    v = mesh.view
    d = _ax_desc(mesh, 5)
    _check(lib().bp_ax_hex3d_f32_multi(ctypes.byref(d), nrhs, mesh.E, v.elementList, v.GlobalToLocal,
                                       _ptr(ops["wJ"]), _ptr(ops["ggeo"]), _ptr(ops["gllw"]), _ptr(ops["D"]),
                                       float(lam), _ptr(q), _ptr(Aq), stream))


OWNER_BIT = 1 << 30


def ogs_owner_map(mesh, out, stream=None):
    """bp_ogs_owner_map: GlobalToLocal of the mesh with OWNER_BIT on the first
    local node of every gathered row, into the int32 device buffer `out`."""
    v = mesh.view
    _check(lib().bp_ogs_owner_map(mesh.NL, v.GlobalToLocal, mesh.Ngather, v.rowStarts, v.colIds, _ptr(out), stream))


def cg_direction_ax(mesh, owner, alpha, beta, r, invD, p_old, p_new, x, Aq, partials, lam=1.0, stream=None):
    """bp_cg_direction_ax_hex3d (FP64): p_new = invD r + beta p_old (beta = 0:
    p_new = invD r), x += alpha p_old (alpha = 0: x untouched), Aq = A_e
    p_new[G2L], p.Ap block partials; invD None means z = r."""
    v = mesh.view
    d = _ax_desc(mesh)
    _check(lib().bp_cg_direction_ax_hex3d(ctypes.byref(d), mesh.E, v.elementList, _ptr(owner), v.wJ, v.ggeo, v.D,
                                          float(lam), float(alpha), float(beta), _ptr(r),
                                          _ptr(invD) if invD is not None else None, _ptr(p_old), _ptr(p_new), _ptr(x),
                                          _ptr(Aq), _ptr(partials), stream))


def cg_direction_ax_f32_multi(mesh, nrhs, owner, ops, alpha, beta, r, invD, p_old, p_new, x, Aq, partials, lam=1.0,
                              stream=None):
    """bp_cg_direction_ax_f32_multi: the fused step in FP32 on nrhs interleaved
    systems; alpha, beta: sequences of nrhs coefficients."""
    v = mesh.view
    d = _ax_desc(mesh, 5)
    a = (ctypes.c_double * nrhs)(*[float(t) for t in alpha])
    b = (ctypes.c_double * nrhs)(*[float(t) for t in beta])
    _check(lib().bp_cg_direction_ax_f32_multi(ctypes.byref(d), nrhs, mesh.E, v.elementList, _ptr(owner),
                                              _ptr(ops["wJ"]), _ptr(ops["ggeo"]), _ptr(ops["D"]), float(lam), a, b,
                                              _ptr(r), _ptr(invD) if invD is not None else None, _ptr(p_old),
                                              _ptr(p_new), _ptr(x), _ptr(Aq), _ptr(partials), stream))


def ogs_gather(mesh, v, gv, stream=None):
    _check(lib().bp_ogs_gather(mesh.Ngather, mesh.view.rowStarts, mesh.view.colIds, _ptr(v), _ptr(gv), stream))


def ogs_scatter(mesh, gv, v, stream=None):
    _check(lib().bp_ogs_scatter(mesh.Ngather, mesh.view.rowStarts, mesh.view.colIds, _ptr(gv), _ptr(v), stream))


NOALLOC_MAX_LOCAL = 1 << 20


def operator_noalloc(mesh, q, Aq, lam=1.0, stream=None, elements=None, nelements=None, nlocal=None):
    """bp_operator_hex3d_noalloc: Aq = Gather(A_e q[G2L]) with no device
    allocation (element results in the library's fixed scratch array), for
    callers that may not call cudaMalloc.  Meshes with E*Np*Nfields above
    NOALLOC_MAX_LOCAL are rejected.  `elements` (a device address of int32
    element ids, `nelements` of them) restricts the operator to a subset of the
    mesh's elements; the default is the whole mesh.  `nlocal` (default: the
    mesh's E*Np*Nfields) is the element-local length the indices must stay
    below."""
    v = mesh.view
    d = _ax_desc(mesh)
    if elements is None:
        elements, nelements = v.elementList, mesh.E
    _check(lib().bp_operator_hex3d_noalloc(ctypes.byref(d), int(nelements), _ptr(elements), v.GlobalToLocal, v.wJ,
                                           v.ggeo, v.gllw, v.D, float(lam), mesh.NL if nlocal is None else int(nlocal),
                                           mesh.Ngather, v.rowStarts,
                                           v.colIds, _ptr(q), _ptr(Aq), stream))


def _ptr(b):
    if isinstance(b, DeviceBuffer):
        return b.ptr
    if isinstance(b, int):
        return b
    raise TypeError("expected a DeviceBuffer or a device address")


class BP:
    """Benchmark problem on a Mesh: bp 1..6 (odd: one field, even: three
    fields, two on a Quad2D mesh; default 5 or 6 by the mesh's field count)."""

    def __init__(self, mesh, bp=None, lam=1.0, precon="NONE", precision="FP64"):
        self.mesh = mesh
        bp = bp or (6 if mesh.Nfields > 1 else 5)
        pc = {"NONE": BP_PRECON_NONE, "JACOBI": BP_PRECON_JACOBI}[precon.upper()]
        pr = {"FP64": BP_PRECISION_FP64, "MIXED": BP_PRECISION_MIXED}[precision.upper()]
        d = SolverDesc(bp, float(lam), pc, pr)
        h = ctypes.c_void_p()
        _check(lib().bp_solver_create(mesh._h, ctypes.byref(d), ctypes.byref(h)))
        self._h = h.value
        self.N = mesh.Ngather
        self.precon = precon.upper()
        self.precision = precision.upper()

    def __del__(self):
        if getattr(self, "_h", None):
            lib().bp_solver_destroy(self._h)
            self._h = None

    def operator(self, q, Aq, stream=None):
        """solver_t::Operator: Aq = Gather(A_e q[G2L]) on device buffers."""
        _check(lib().bp_solver_operator(self._h, _ptr(q), _ptr(Aq), stream))

    def rhs(self, mode="ANALYTIC", seed=0, b=None, f=None):
        """Gathered forcing into a device buffer (returned)."""
        b = b or DeviceBuffer(self.N)
        m = {"ANALYTIC": BP_RHS_ANALYTIC, "RANDOM": BP_RHS_RANDOM}[mode.upper()]
        _check(lib().bp_solver_rhs(self._h, m, int(seed), b.ptr, f.ptr if f is not None else None))
        return b

    def diagonal(self):
        d = DeviceBuffer(self.N)
        _check(lib().bp_solver_diagonal(self._h, d.ptr))
        return d

    def solve(self, x, r, tol=0.0, maxit=100, history=True):
        """cg::Solve on device buffers (x in/out, r = b in / residual out).
        Returns (stats, rnorm_history, alpha_history)."""
        st = SolveStats()
        hr = np.zeros(max(maxit, 1))
        ha = np.zeros(max(maxit, 1))
        _check(lib().bp_solver_solve(self._h, x.ptr, r.ptr, float(tol), int(maxit),
                                     hr.ctypes.data if history else None, ha.ctypes.data if history else None,
                                     ctypes.byref(st)))
        it = st.iterations
        return st, hr[:it], ha[:it]

    def solve_host(self, b_host, x_host, tol=0.0, maxit=100):
        """The same solve from host arrays (copies inside the call)."""
        st = SolveStats()
        b_host = np.ascontiguousarray(b_host, dtype=np.float64)
        assert x_host.dtype == np.float64 and x_host.flags.c_contiguous
        _check(lib().bp_solver_solve_host(self._h, b_host.ctypes.data, x_host.ctypes.data, float(tol), int(maxit),
                                          ctypes.byref(st)))
        return st


class Batch:
    """Many independent problems with several right-hand sides each, solved
    together (bp_batch_*).  problems: iterable of dicts with nx, ny, nz, N,
    pert, pert_seed, nrhs, rhs_seed."""

    def __init__(self, problems, bp=5, lam=1.0, precon="JACOBI", precision="MIXED"):
        platform_init(0)
        probs = list(problems)
        arr = (BatchProblem * len(probs))(*[
            BatchProblem(p["nx"], p.get("ny", p["nx"]), p.get("nz", p["nx"]), p["N"], float(p.get("pert", 0.0)),
                         int(p.get("pert_seed", 1)), int(p.get("nrhs", 1)), int(p.get("rhs_seed", 0)),
                         int(bool(p.get("affine", False))))
            for p in probs])
        pc = {"NONE": BP_PRECON_NONE, "JACOBI": BP_PRECON_JACOBI}[precon.upper()]
        pr = {"FP64": BP_PRECISION_FP64, "MIXED": BP_PRECISION_MIXED}[precision.upper()]
        d = SolverDesc(bp, float(lam), pc, pr)
        h = ctypes.c_void_p()
        _check(lib().bp_batch_create(arr, len(probs), ctypes.byref(d), ctypes.byref(h)))
        self._h = h.value
        n = ctypes.c_int32()
        _check(lib().bp_batch_systems(self._h, ctypes.byref(n)))
        self.nsystems = n.value
        self.problem, self.Ngather = [], []
        for s in range(self.nsystems):
            pj, ng = ctypes.c_int32(), ctypes.c_int32()
            _check(lib().bp_batch_system_info(self._h, s, ctypes.byref(pj), ctypes.byref(ng)))
            self.problem.append(pj.value)
            self.Ngather.append(ng.value)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().bp_batch_destroy(self._h)
            self._h = None

    def solve(self, tol=1e-8, maxit=5000):
        """Solve every system; returns (list of SolveStats, device ms)."""
        st = (SolveStats * self.nsystems)()
        ms = ctypes.c_double()
        _check(lib().bp_batch_solve(self._h, float(tol), int(maxit), st, ctypes.byref(ms)))
        return list(st), ms.value

    def vectors(self, system):
        """(x, b) of a system copied to the host."""
        xp, bp_ = ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib().bp_batch_vectors(self._h, system, ctypes.byref(xp), ctypes.byref(bp_)))
        n = self.Ngather[system]
        return _dl(xp.value, n, np.float64), _dl(bp_.value, n, np.float64)

    def operator(self, system, q, Aq):
        """The system's operator (bp_solver_operator) on device buffers."""
        sv = ctypes.c_void_p()
        _check(lib().bp_batch_solver(self._h, system, ctypes.byref(sv)))
        _check(lib().bp_solver_operator(sv.value, _ptr(q), _ptr(Aq), None))


def lcg_uniform(seed, n):
    """n draws of the reference's seeded LCG (libs/primitives/random.cpp): the
    state starts at a*(~seed)+1 and each value is state/(2^64-1) before the
    step.  Host-side, for generating problem sets."""
    a, mask = 6364136223846793005, (1 << 64) - 1
    x = (a * (mask ^ (seed & mask)) + 1) & mask
    out = []
    for _ in range(n):
        out.append(float(x) / float(mask))
        x = (a * x + 1) & mask
    return out


def uneven_problems(count=64, seed=2, nrhs=4, pmin=3, pmax=10, nmin=8, nmax=24, pert=0.1):
    """The batched problem set: problem i has degree p_i = pmin + floor(u_{2i}
    (pmax-pmin+1)) and n_i = nmin + floor(u_{2i+1} (nmax-nmin+1)) elements per
    side (draws u of the LCG with `seed`), interior vertices perturbed by
    pert*h (seed 100+i), and nrhs right-hand sides with seeds 1000+nrhs*i+k."""
    u = lcg_uniform(seed, 2 * count)
    probs = []
    for i in range(count):
        p = pmin + min(int(u[2 * i] * (pmax - pmin + 1)), pmax - pmin)
        n = nmin + min(int(u[2 * i + 1] * (nmax - nmin + 1)), nmax - nmin)
        probs.append({"nx": n, "N": p, "pert": pert, "pert_seed": 100 + i, "nrhs": nrhs, "rhs_seed": 1000 + nrhs * i})
    return probs


def box_numbering(nx, ny, nz, N, Nfields=1, dim=3, simplex=False):
    """Host-only masked numbering of the box: (GlobalToLocal, rowStarts, colIds).
    dim=2: the Quad2D box of nx x ny elements (nz ignored); with simplex=True
    the Tri2D box of 2 nx ny triangles."""
    d = BoxDesc(nx, ny, nz if dim == 3 else 1, N, int(bool(simplex)), Nfields, 0.0, 1, dim, int(bool(simplex)))
    ng, nnz = ctypes.c_int32(), ctypes.c_int32()
    _check(lib().bp_box_numbering(ctypes.byref(d), ctypes.byref(ng), ctypes.byref(nnz), None, None, None))
    E = nx * ny * (nz if dim == 3 else 1) * ((2 if dim == 2 else 6) if simplex else 1)
    if simplex:
        Np = (N + 1) * (N + 2) // 2 if dim == 2 else (N + 1) * (N + 2) * (N + 3) // 6
    else:
        Np = (N + 1) ** dim
    g2l = np.empty(E * Np * Nfields, np.int32)
    rs = np.empty(ng.value + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    _check(lib().bp_box_numbering(ctypes.byref(d), None, None, g2l.ctypes.data, rs.ctypes.data, ci.ctypes.data))
    return g2l, rs, ci


def basis_tri2d(N):
    """Host-only Tri2D reference element: r, s [Np], Dr, Ds, MM, Srr, Srs, Sss as
    row-major Np x Np arrays (X[n, k] weighs node k in output n)."""
    Np = (N + 1) * (N + 2) // 2
    r, s = np.empty(Np), np.empty(Np)
    D, MM, S = np.empty(2 * Np * Np), np.empty(Np * Np), np.empty(3 * Np * Np)
    _check(lib().bp_basis_tri2d(N, r.ctypes.data, s.ctypes.data, D.ctypes.data, MM.ctypes.data, S.ctypes.data))
    D = D.reshape(2, Np, Np).transpose(0, 2, 1)
    S = S.reshape(3, Np, Np).transpose(0, 2, 1)
    return r, s, D[0], D[1], MM.reshape(Np, Np), S[0], S[1], S[2]


def basis_tet3d(N):
    """Host-only Tet3D reference element: r, s, t [Np], Dr, Ds, Dt, MM and S [6]
    (rr, rs, rt, ss, st, tt) as row-major Np x Np arrays."""
    Np = (N + 1) * (N + 2) * (N + 3) // 6
    r, s, t = np.empty(Np), np.empty(Np), np.empty(Np)
    D, MM, S = np.empty(3 * Np * Np), np.empty(Np * Np), np.empty(6 * Np * Np)
    _check(lib().bp_basis_tet3d(N, r.ctypes.data, s.ctypes.data, t.ctypes.data, D.ctypes.data, MM.ctypes.data,
                                S.ctypes.data))
    D = D.reshape(3, Np, Np).transpose(0, 2, 1)
    S = S.reshape(6, Np, Np).transpose(0, 2, 1)
    return r, s, t, D[0], D[1], D[2], MM.reshape(Np, Np), S


def basis_gll(N):
    """Host-only GLL nodes, weights and differentiation matrix of degree N."""
    z = np.empty(N + 1); w = np.empty(N + 1); D = np.empty((N + 1) * (N + 1))
    _check(lib().bp_basis_gll(N, z.ctypes.data, w.ctypes.data, D.ctypes.data))
    return z, w, D.reshape(N + 1, N + 1)


def basis_cubature(N):
    """Host-only cubature data of degree N: dict of r, w (N+2), I [(N+2) x (N+1)],
    D [(N+2) x (N+2)], invV, Dmodal, MM [(N+1) x (N+1)]."""
    G, Nq = N + 2, N + 1
    out = {"r": np.empty(G), "w": np.empty(G), "I": np.empty(G * Nq), "D": np.empty(G * G),
           "invV": np.empty(Nq * Nq), "Dmodal": np.empty(Nq * Nq), "MM": np.empty(Nq * Nq)}
    _check(lib().bp_basis_cubature(N, *(out[k].ctypes.data for k in ("r", "w", "I", "D", "invV", "Dmodal", "MM"))))
    out["I"] = out["I"].reshape(G, Nq)
    out["D"] = out["D"].reshape(G, G)
    for k in ("invV", "Dmodal", "MM"):
        out[k] = out[k].reshape(Nq, Nq)
    return out


FORMS = {0: "mma", 1: "tma", 2: "line", 3: "pencil", 4: "rb"}


def tune_report(kind, N, Nfields, affine, precision_bytes, lanes, fused, Nelements):
    """(chosen form name or None, {form name: ms}) for an element-operator configuration."""
    f, n = ctypes.c_int32(), ctypes.c_int32()
    forms = np.zeros(8, np.int32)
    ms = np.zeros(8, np.float32)
    _check(lib().bp_tune_report(kind, N, Nfields, int(affine), precision_bytes, lanes, int(fused), Nelements,
                                ctypes.byref(f), ctypes.byref(n), forms.ctypes.data, ms.ctypes.data, 8))
    return (FORMS.get(f.value), {FORMS[int(forms[k])]: float(ms[k]) for k in range(n.value)})


def tune_reset():
    _check(lib().bp_tune_reset())


def ogs_check(g2l, rowStarts, colIds, Ngather):
    """bp_ogs_check on host arrays: raises BPError naming the first broken rule."""
    g = np.ascontiguousarray(g2l, dtype=np.int32)
    rs = np.ascontiguousarray(rowStarts, dtype=np.int32)
    ci = np.ascontiguousarray(colIds, dtype=np.int32)
    _check(lib().bp_ogs_check(g.size, g.ctypes.data, int(Ngather), rs.ctypes.data, ci.ctypes.data))


def box_vertices(nx, ny, nz, pert=0.0, pert_seed=1, dim=3):
    """Host-only vertex coordinates (EX, EY, EZ), each [E*8]; dim=2: (EX, EY)
    of the Quad2D box, each [E*4], and an empty EZ."""
    d = BoxDesc(nx, ny, nz if dim == 3 else 1, 1, 0, 1, float(pert), int(pert_seed), dim)
    if dim == 2:
        E = nx * ny
        ex, ey = np.empty(4 * E), np.empty(4 * E)
        _check(lib().bp_box_vertices(ctypes.byref(d), ex.ctypes.data, ey.ctypes.data, None))
        return ex, ey, np.empty(0)
    E = nx * ny * nz
    ex, ey, ez = (np.empty(8 * E) for _ in range(3))
    _check(lib().bp_box_vertices(ctypes.byref(d), ex.ctypes.data, ey.ctypes.data, ez.ctypes.data))
    return ex, ey, ez


def driver_main(name, args):
    """Run a BK/BP executable's main() in-process (e.g. driver_main("BP5", ["-nx","8"]))."""
    argv = [name.encode()] + [a.encode() for a in args]
    arr = (ctypes.c_char_p * len(argv))(*argv)
    return lib().bp_driver_main(name.encode(), len(argv), arr)
