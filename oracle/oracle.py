"""ctypes wrapper of the CPU oracle (oracle/bp_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg as the checker.  The product package never imports
this module.

The oracle restates the reference's Hex3D (and Quad2D BP5/BP6) BK/BP hot path
on the CPU (see the header of bp_oracle.cpp for the reference file:line of
every routine).

Parity pin: the reference's own host set-up code, compiled here against
host-only shims (oracle/Makefile, target ref), produced the fixtures of
tests/golden/, which tests/test_ref_golden.py holds this restatement to; the
element kernels (OKL, which need OCCA) are pinned by known answers of the
mathematics (tests/test_oracle.py, tests/test_cub_host.py).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libbp_oracle.so")
_lib = None

_c_dp = ctypes.POINTER(ctypes.c_double)


def build():
    """Compile libbp_oracle.so with oracle/Makefile."""
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.bpo_random.argtypes = [ctypes.c_uint64, ctypes.c_int64, _c_dp]
        L.bpo_jacobi_gq.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, _c_dp, _c_dp]
        L.bpo_jacobi_gll.argtypes = [ctypes.c_int, _c_dp, _c_dp]
        L.bpo_dmatrix1d.argtypes = [ctypes.c_int, _c_dp, ctypes.c_int, _c_dp, _c_dp]
        L.bpo_interp_matrix1d.argtypes = [ctypes.c_int, _c_dp, ctypes.c_int, _c_dp, _c_dp]
        L.bpo_mass_matrix1d.argtypes = [ctypes.c_int, _c_dp, _c_dp]
        L.bpo_mesh_create.restype = ctypes.c_void_p
        L.bpo_mesh_create.argtypes = [ctypes.c_int] * 6 + [ctypes.c_double, ctypes.c_uint64]
        L.bpo_mesh_create2d.restype = ctypes.c_void_p
        L.bpo_mesh_create2d.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double, ctypes.c_uint64]
        L.bpo_mesh_free.argtypes = [ctypes.c_void_p]
        L.bpo_mesh_int.restype = ctypes.c_int64
        L.bpo_mesh_int.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.bpo_mesh_array.restype = ctypes.c_void_p
        L.bpo_mesh_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        L.bpo_ax_bp5.argtypes = [ctypes.c_void_p, ctypes.c_double, _c_dp, _c_dp]
        L.bpo_gather.argtypes = [ctypes.c_void_p, _c_dp, _c_dp]
        L.bpo_scatter.argtypes = [ctypes.c_void_p, _c_dp, _c_dp]
        L.bpo_operator_bp5.argtypes = [ctypes.c_void_p, ctypes.c_double, _c_dp, _c_dp]
        L.bpo_rhs_analytic.argtypes = [ctypes.c_void_p, ctypes.c_double, _c_dp]
        L.bpo_rhs_random.argtypes = [ctypes.c_void_p, ctypes.c_uint64, _c_dp, _c_dp]
        L.bpo_jacobi_diag_bp5.argtypes = [ctypes.c_void_p, ctypes.c_double, _c_dp]
        L.bpo_cg.restype = ctypes.c_int
        L.bpo_cg.argtypes = [ctypes.c_void_p, ctypes.c_double, _c_dp, _c_dp, ctypes.c_double,
                             ctypes.c_int, ctypes.c_int, _c_dp, _c_dp, _c_dp]
        L.bpo_ax.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _c_dp, _c_dp]
        L.bpo_operator.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _c_dp, _c_dp]
        L.bpo_jacobi_diag.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _c_dp]
        L.bpo_cg_bp.restype = ctypes.c_int
        L.bpo_cg_bp.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _c_dp, _c_dp, ctypes.c_double,
                                ctypes.c_int, ctypes.c_int, _c_dp, _c_dp, _c_dp]
        L.bpo_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_c_dp)


def random(seed, n):
    """prim::seedRNG(seed) followed by prim::random<double>(n)."""
    v = np.empty(n, dtype=np.float64)
    lib().bpo_random(seed, n, _dp(v))
    return v


def jacobi_gll(N):
    x = np.empty(N + 1); w = np.empty(N + 1)
    assert lib().bpo_jacobi_gll(N, _dp(x), _dp(w)) == 0
    return x, w


def jacobi_gq(alpha, beta, N):
    x = np.empty(N + 1); w = np.empty(N + 1)
    assert lib().bpo_jacobi_gq(alpha, beta, N, _dp(x), _dp(w)) == 0
    return x, w


def dmatrix1d(N, rin, rout):
    rin = np.ascontiguousarray(rin, dtype=np.float64)
    rout = np.ascontiguousarray(rout, dtype=np.float64)
    D = np.empty((len(rout), N + 1))
    assert lib().bpo_dmatrix1d(N, _dp(rin), len(rout), _dp(rout), _dp(D)) == 0
    return D


def interp_matrix1d(N, rin, rout):
    rin = np.ascontiguousarray(rin, dtype=np.float64)
    rout = np.ascontiguousarray(rout, dtype=np.float64)
    I = np.empty((len(rout), N + 1))
    assert lib().bpo_interp_matrix1d(N, _dp(rin), len(rout), _dp(rout), _dp(I)) == 0
    return I


_DTYPES = {
    "gllz": np.float64, "gllw": np.float64, "D": np.float64, "MM": np.float64,
    "EToV": np.int64, "EX": np.float64, "EY": np.float64, "EZ": np.float64,
    "EToE": np.int32, "globalIds": np.int64, "x": np.float64, "y": np.float64,
    "z": np.float64, "wJ": np.float64, "ggeo": np.float64, "maskedIds": np.int64,
    "rowStarts": np.int32, "colIds": np.int32, "G2L": np.int32,
    "blockRowStarts": np.int32, "elementList": np.int32,
    "cubr": np.float64, "cubw": np.float64, "cubInterp": np.float64, "cubD": np.float64,
    "invV": np.float64, "cubwJ": np.float64, "cubggeo": np.float64,
}


class Mesh:
    """Box mesh with masked ogs numbering, built by the oracle.

    nx, ny, nz: elements per direction; N: degree; affine: store per-element
    factors; Nfields: 1 (BP5) or 3 (BP6; 2 in 2D); pert/pert_seed: seeded
    perturbation of interior vertices by pert*h*(2u-1).  dim=2 builds the
    Quad2D box of nx x ny elements (nz is ignored; BP5/BP6 only)."""

    def __init__(self, nx, ny, nz, N, affine=False, Nfields=1, pert=0.0, pert_seed=1, dim=3):
        if dim == 2:
            self._h = lib().bpo_mesh_create2d(nx, ny, N, int(bool(affine)), Nfields, float(pert), pert_seed)
        else:
            self._h = lib().bpo_mesh_create(nx, ny, nz, N, int(bool(affine)), Nfields, float(pert), pert_seed)
        if not self._h:
            raise RuntimeError("oracle mesh setup failed (bad sizes or non-positive Jacobian)")
        self.dim = dim
        self.nx, self.ny, self.nz, self.N = nx, ny, (nz if dim == 3 else 1), N
        self.affine = bool(affine)
        self.Nfields = Nfields
        for k in ("Nq", "Np", "E", "Ngather", "nnz"):
            setattr(self, k, int(lib().bpo_mesh_int(self._h, k.encode())))
        self._cache = {}

    def __del__(self):
        if getattr(self, "_h", None):
            lib().bpo_mesh_free(self._h)
            self._h = None

    def array(self, name):
        """A copy of a named mesh array (see _DTYPES for names)."""
        if name not in self._cache:
            n = ctypes.c_int64(0)
            ptr = lib().bpo_mesh_array(self._h, name.encode(), ctypes.byref(n))
            if n.value < 0:
                raise KeyError(name)
            if n.value == 0:
                self._cache[name] = np.empty(0, dtype=_DTYPES[name])
            else:
                ct = np.ctypeslib.as_ctypes_type(_DTYPES[name])
                buf = (ct * n.value).from_address(ptr)
                self._cache[name] = np.frombuffer(buf, dtype=_DTYPES[name]).copy()
        return self._cache[name]

    @property
    def NL(self):
        return self.E * self.Np * self.Nfields

    def ax(self, q, lam=1.0, bp=5):
        """Element-local operator AqL = A_e q[G2L] of benchmark problem bp:
        1/2 mass, 3/4 over-integrated stiffness, 5/6 collocated stiffness
        (the field count comes from the mesh)."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        out = np.empty(self.NL)
        if self.dim == 2 and bp < 5:
            raise ValueError("the oracle's Quad2D forms are BP5/BP6")
        if bp >= 5:
            lib().bpo_ax_bp5(self._h, lam, _dp(q), _dp(out))
        else:
            lib().bpo_ax(self._h, bp, lam, _dp(q), _dp(out))
        return out

    def gather(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        out = np.empty(self.Ngather)
        lib().bpo_gather(self._h, _dp(v), _dp(out))
        return out

    def scatter(self, gv, fill=0.0):
        gv = np.ascontiguousarray(gv, dtype=np.float64)
        out = np.full(self.NL, fill)
        lib().bpo_scatter(self._h, _dp(gv), _dp(out))
        return out

    def operator(self, q, lam=1.0, bp=5):
        if self.dim == 2 and bp < 5:
            raise ValueError("the oracle's Quad2D forms are BP5/BP6")
        q = np.ascontiguousarray(q, dtype=np.float64)
        out = np.empty(self.Ngather)
        lib().bpo_operator(self._h, bp, lam, _dp(q), _dp(out))
        return out

    def rhs_analytic(self, lam=1.0):
        """Gathered analytic forcing b = Gather(wJ f(x,y,z))."""
        rL = np.empty(self.NL)
        lib().bpo_rhs_analytic(self._h, lam, _dp(rL))
        return self.gather(rL)

    def rhs_random(self, seed=0):
        """Seeded nodal forcing f = 2u-1 and b = M f.  Returns (f, b)."""
        f = np.empty(self.Ngather); b = np.empty(self.Ngather)
        lib().bpo_rhs_random(self._h, seed, _dp(f), _dp(b))
        return f, b

    def jacobi_diag(self, lam=1.0, bp=5):
        d = np.empty(self.Ngather)
        lib().bpo_jacobi_diag(self._h, bp, lam, _dp(d))
        return d

    def cg(self, b, lam=1.0, tol=0.0, maxit=100, precon=False, x0=None, bp=5):
        """cg::Solve.  Returns (x, r_final, iterations, rnorm_history, alpha_history)."""
        x = np.zeros(self.Ngather) if x0 is None else np.array(x0, dtype=np.float64)
        r = np.array(b, dtype=np.float64)
        hr = np.zeros(maxit); ha = np.zeros(maxit)
        inv = None
        if precon:
            inv = 1.0 / self.jacobi_diag(lam, bp)
        it = lib().bpo_cg_bp(self._h, bp, lam, _dp(x), _dp(r), tol, maxit, int(bool(precon)), _dp(inv),
                             _dp(hr), _dp(ha))
        return x, r, it, hr[:it], ha[:it]


def num_threads():
    return int(lib().bpo_num_threads())
