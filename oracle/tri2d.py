"""CPU restatement of the reference's Tri2D BP5 path (numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the library's
Tri2D meshes and operators; the product package never imports it.

What it restates (reference files, paths relative to the reference root):
  nodes        equispaced (r, s) rows (libs/mesh/meshBasisTri2D.cpp:200-217)
               warped and blended (Warburton 2006; :509-585, alpha table of
               :517-518) with the warp factor interpolated from equispaced to
               GLL nodes (:461-488)
  matrices     Vandermonde of an orthonormal basis of P_N, Dr = Vr V^-1,
               Ds = Vs V^-1, MM = (V V^T)^-1 (meshReferenceNodesTri2D.cpp:41-52),
               Srr = Dr^T MM Dr, Srs = Dr^T MM Ds + Ds^T MM Dr,
               Sss = Ds^T MM Ds (meshBasisTri2D.cpp:406-430).  Dr, Ds, MM and S
               do not depend on which basis of P_N builds V; the orthonormal
               Koornwinder-Dubiner basis keeps V well conditioned.
  box          two triangles per box cell (meshSetupBoxTri2D.cpp:78-107)
  geometry     affine factors per element: J, G00 = J(rx^2+ry^2),
               G01 = J(rx sx + ry sy), G11 = J(sx^2+sy^2)
               (meshGeometricFactorsTri2D.cpp)
  numbering    the global id of a node is the smallest 1 + e*Np + n over its
               copies (meshConnectNodes.cpp:32-82); the copies on boundary
               faces are masked, copy by copy, so a boundary vertex stays live
               through the copies of elements that touch it only at that vertex
               (meshMaskedGatherScatterSetup.cpp:31-56); gathered rows in the
               order of each node's first unmasked local copy, each row's
               local columns ascending (ogsSetup.cpp)
  operator     AqL_e = G00 Srr q_e + G01 Srs q_e + G11 Sss q_e + lambda J MM q_e
               (okl/bp5AxAffineTri2D.okl:27-89)
  forcing      b = Gather(J MM f_e) of a seeded nodal f = 2u - 1, or the
               analytic forcing of okl/rhsTri2D.okl (rhsAffineTri2D)
  CG           the reference's cg::Solve with optional Jacobi (as the Hex3D oracle)

Parity pin: tests/golden/ref_tri_*.npz, written by the reference's own set-up
code (tests/golden/make_golden.py), hold the node coordinates, D, MM, S, the
geometric factors, the numbering, the CSR and the host gather/scatter that
tests/test_tri2d.py compares this restatement to.
"""
import numpy as np
from threadpoolctl import threadpool_limits

from oracle import oracle as _o

# One BLAS thread for the dense inverses and products here: a threaded BLAS
# pool next to torch's OpenMP runtime in the same test process has deadlocked
# in np.linalg.inv.
threadpool_limits(limits=1, user_api="blas")

ALPHA_OPT = [0.0000, 0.0000, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999, 1.2832, 1.3648, 1.4773, 1.4959, 1.5743,
             1.5770, 1.6223, 1.6258]


def _lagrange(xn, x):
    """Values of the Lagrange polynomials on nodes xn at points x: [len(x), len(xn)]."""
    L = np.ones((len(x), len(xn)))
    for j, xj in enumerate(xn):
        for m, xm in enumerate(xn):
            if m != j:
                L[:, j] *= (x - xm) / (xj - xm)
    return L


def _warp(N, r):
    gll = np.asarray(_o.jacobi_gll(N)[0], dtype=np.float64)
    req = -1.0 + 2.0 * np.arange(N + 1) / N
    w = _lagrange(req, r) @ (gll - req)
    inside = np.abs(r) < 1.0 - 1.0e-10
    sf = 1.0 - (inside * r) ** 2
    return w / sf + w * (inside - 1.0)


def nodes(N):
    """Warp & blend nodes (r, s) in the reference's order."""
    r, s = [], []
    for n in range(N + 1):
        for m in range(N + 1 - n):
            r.append(-1.0 + 2.0 * m / N)
            s.append(-1.0 + 2.0 * n / N)
    r, s = np.array(r), np.array(s)
    alpha = ALPHA_OPT[N - 1] if N < 16 else 5.0 / 3.0
    L1, L2, L3 = 0.5 * (1 + s), -0.5 * (r + s), 0.5 * (1 + r)
    x = -L2 + L3
    y = (-L2 - L3 + 2 * L1) / np.sqrt(3.0)
    w1 = 4 * L2 * L3 * _warp(N, L3 - L2) * (1 + (alpha * L1) ** 2)
    w2 = 4 * L3 * L1 * _warp(N, L1 - L3) * (1 + (alpha * L2) ** 2)
    w3 = 4 * L1 * L2 * _warp(N, L2 - L1) * (1 + (alpha * L3) ** 2)
    x = x + w1 + np.cos(2 * np.pi / 3) * w2 + np.cos(4 * np.pi / 3) * w3
    y = y + np.sin(2 * np.pi / 3) * w2 + np.sin(4 * np.pi / 3) * w3
    l1 = (np.sqrt(3.0) * y + 1) / 3
    l2 = (-3 * x - np.sqrt(3.0) * y + 2) / 6
    l3 = (3 * x - np.sqrt(3.0) * y + 2) / 6
    return -l2 + l3 - l1, -l2 - l3 + l1


def _jacobi(x, a, b, n):
    """Orthonormal Jacobi polynomial P_n^(a,b) at x and its derivative."""
    x = np.asarray(x, dtype=np.float64)
    from math import gamma
    g0 = 2 ** (a + b + 1) / (a + b + 1) * gamma(a + 1) * gamma(b + 1) / gamma(a + b + 1)
    P = [np.full_like(x, 1.0 / np.sqrt(g0))]
    if n > 0:
        g1 = (a + 1) * (b + 1) / (a + b + 3) * g0
        P.append(((a + b + 2) * x / 2 + (a - b) / 2) / np.sqrt(g1))
    aold = 2 / (2 + a + b) * np.sqrt((a + 1) * (b + 1) / (a + b + 3))
    for i in range(1, n):
        h1 = 2 * i + a + b
        anew = 2 / (h1 + 2) * np.sqrt((i + 1) * (i + 1 + a + b) * (i + 1 + a) * (i + 1 + b) / (h1 + 1) / (h1 + 3))
        bnew = -(a * a - b * b) / h1 / (h1 + 2)
        P.append(1 / anew * (-aold * P[i - 1] + (x - bnew) * P[i]))
        aold = anew
    val = P[n]
    if n == 0:
        dval = np.zeros_like(x)
    else:
        dval = np.sqrt(n * (n + a + b + 1)) * _jacobi(x, a + 1, b + 1, n - 1)[0]
    return val, dval


def vandermonde(N, r, s):
    """V, Vr, Vs of the orthonormal basis sqrt(2) P_i(a) P_j^(2i+1,0)(b) (1-b)^i."""
    r, s = np.asarray(r), np.asarray(s)
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(s != 1.0, 2 * (1 + r) / (1 - s) - 1, -1.0)
    b = s
    cols, cr, cs = [], [], []
    for i in range(N + 1):
        for j in range(N + 1 - i):
            fa, dfa = _jacobi(a, 0, 0, i)
            gb, dgb = _jacobi(b, 2 * i + 1, 0, j)
            cols.append(np.sqrt(2.0) * fa * gb * (1 - b) ** i)
            # d/dr = da/dr d/da, d/ds = da/ds d/da + d/db (a and b as above)
            dmodedr = dfa * gb
            if i > 0:
                dmodedr = dmodedr * (0.5 * (1 - b)) ** (i - 1)
            dmodeds = dfa * (gb * (0.5 * (1 + a)))
            if i > 0:
                dmodeds = dmodeds * (0.5 * (1 - b)) ** (i - 1)
            tmp = dgb * (0.5 * (1 - b)) ** i
            if i > 0:
                tmp = tmp - 0.5 * i * gb * (0.5 * (1 - b)) ** (i - 1)
            dmodeds = dmodeds + fa * tmp
            cr.append(2 ** (i + 0.5) * dmodedr)
            cs.append(2 ** (i + 0.5) * dmodeds)
    return np.array(cols).T, np.array(cr).T, np.array(cs).T


def reference_matrices(N):
    """r, s, Dr, Ds, MM, Srr, Srs, Sss (row-major: X[n, m] acts on node m for output n)."""
    r, s = nodes(N)
    V, Vr, Vs = vandermonde(N, r, s)
    Vi = np.linalg.inv(V)
    Dr, Ds = Vr @ Vi, Vs @ Vi
    MM = np.linalg.inv(V @ V.T)
    Srr = Dr.T @ MM @ Dr
    Srs = Dr.T @ MM @ Ds + Ds.T @ MM @ Dr
    Sss = Ds.T @ MM @ Ds
    return r, s, Dr, Ds, MM, Srr, Srs, Sss


class Mesh:
    """The Tri2D box [-1,1]^2 of nx*ny cells, two triangles each, degree N."""

    def __init__(self, nx, ny, N):
        self.nx, self.ny, self.N = nx, ny, N
        self.Np = (N + 1) * (N + 2) // 2
        self.E = 2 * nx * ny
        (self.r, self.s, self.Dr, self.Ds, self.MM, self.Srr, self.Srs, self.Sss) = reference_matrices(N)
        # box vertices (format of meshSetupBoxTri2D.cpp:78-107)
        dx, dy = 2.0 / nx, 2.0 / ny
        NnX = nx + 1
        EToV, EX, EY = [], [], []
        for j in range(ny):
            for i in range(nx):
                x0, y0 = -1.0 + dx * i, -1.0 + dy * j
                v00, v10, v11, v01 = i + j * NnX, (i + 1) + j * NnX, (i + 1) + (j + 1) * NnX, i + (j + 1) * NnX
                EToV += [v00, v10, v11, v00, v11, v01]
                EX += [x0, x0 + dx, x0 + dx, x0, x0 + dx, x0]
                EY += [y0, y0, y0 + dy, y0, y0 + dy, y0 + dy]
        self.EToV = np.array(EToV, np.int64)
        self.EX, self.EY = np.array(EX), np.array(EY)
        ex, ey = self.EX.reshape(-1, 3), self.EY.reshape(-1, 3)
        r, s = self.r, self.s
        self.x = (-(r + s)[None, :] * ex[:, :1] + (1 + r)[None, :] * ex[:, 1:2] + (1 + s)[None, :] * ex[:, 2:3]) / 2
        self.y = (-(r + s)[None, :] * ey[:, :1] + (1 + r)[None, :] * ey[:, 1:2] + (1 + s)[None, :] * ey[:, 2:3]) / 2
        # affine geometric factors per element
        xr, xs = (ex[:, 1] - ex[:, 0]) / 2, (ex[:, 2] - ex[:, 0]) / 2
        yr, ys = (ey[:, 1] - ey[:, 0]) / 2, (ey[:, 2] - ey[:, 0]) / 2
        J = xr * ys - xs * yr
        rx, ry, sx, sy = ys / J, -xs / J, -yr / J, xr / J
        self.wJ = J
        self.ggeo = np.stack([J * (rx * rx + ry * ry), J * (rx * sx + ry * sy), J * (sx * sx + sy * sy)], axis=1)
        self._number()

    def _number(self):
        # node identity by position (shared copies coincide to rounding), id =
        # min over copies of 1 + e*Np + n, boundary nodes masked
        Np, E = self.Np, self.E
        key = np.round(np.stack([self.x.ravel(), self.y.ravel()], axis=1) * 1e9).astype(np.int64)
        _, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.ravel()
        lid = np.arange(E * Np)
        gmin = np.full(inv.max() + 1, np.iinfo(np.int64).max)
        np.minimum.at(gmin, inv, lid + 1)
        self.globalIds = gmin[inv]
        # masking is per copy: the copies on an element's boundary faces
        # (faces 0, 1, 2: s = -1, r + s = 0, r = -1) are masked, other copies of
        # the same node (through a boundary vertex) are not, as in the
        # reference's mesh_t::MaskedGatherScatterSetup
        tol = 1e-5
        fnodes = [np.flatnonzero(np.abs(self.s + 1) < tol), np.flatnonzero(np.abs(self.r + self.s) < tol),
                  np.flatnonzero(np.abs(self.r + 1) < tol)]
        fverts = [(0, 1), (1, 2), (2, 0)]
        ex, ey = self.EX.reshape(-1, 3), self.EY.reshape(-1, 3)
        masked = np.zeros(E * Np, bool)
        for e in range(E):
            for f, (a, b) in enumerate(fverts):
                on = any(abs(c[e, a] - v) < 1e-12 and abs(c[e, b] - v) < 1e-12 for c in (ex, ey) for v in (-1.0, 1.0))
                if on:
                    masked[e * Np + fnodes[f]] = True
        # rows in the order of each node's first unmasked copy (for a node
        # whose lowest copy is unmasked this is its global id's order)
        row = {}
        for l in np.flatnonzero(~masked):
            row.setdefault(self.globalIds[l], len(row))
        live = list(row)
        self.G2L = np.array([-1 if masked[l] else row[self.globalIds[l]] for l in range(E * Np)], np.int32)
        self.Ngather = len(live)
        cols = [[] for _ in range(self.Ngather)]
        for l in range(E * Np):
            if self.G2L[l] >= 0:
                cols[self.G2L[l]].append(l)
        self.rowStarts = np.zeros(self.Ngather + 1, np.int32)
        self.rowStarts[1:] = np.cumsum([len(c) for c in cols])
        self.colIds = np.array([c for cs in cols for c in cs], np.int32)

    @property
    def NL(self):
        return self.E * self.Np

    def scatter(self, g):
        return np.where(self.G2L >= 0, np.asarray(g)[np.maximum(self.G2L, 0)], 0.0)

    def gather(self, v):
        v = np.asarray(v)
        out = np.zeros(self.Ngather)
        for k in range(self.Ngather):
            acc = 0.0
            for c in self.colIds[self.rowStarts[k]:self.rowStarts[k + 1]]:
                acc += v[c]
            out[k] = acc
        return out

    def ax(self, q, lam=1.0):
        """Element-local AqL for a gathered q, in the reference kernel's order of sums."""
        qL = self.scatter(q).reshape(self.E, self.Np)
        g = self.ggeo
        out = np.empty_like(qL)
        for e in range(self.E):
            qrr = self.Srr @ qL[e]
            qrs = self.Srs @ qL[e]
            qss = self.Sss @ qL[e]
            qM = self.MM @ qL[e]
            out[e] = g[e, 0] * qrr + g[e, 1] * qrs + g[e, 2] * qss + self.wJ[e] * lam * qM
        return out.ravel()

    def operator(self, q, lam=1.0):
        return self.gather(self.ax(q, lam))

    def rhs_random(self, seed=0):
        f = 2.0 * _o.random(seed, self.Ngather) - 1.0
        fL = self.scatter(f).reshape(self.E, self.Np)
        bL = (self.wJ[:, None] * (fL @ self.MM.T)).ravel()
        return f, self.gather(bL)

    def rhs_analytic(self, lam=1.0):
        """rhsAffineTri2D (okl/rhsTri2D.okl): Gather(MM (J f)) with
        f = (2 pi^2 + lambda) sin(pi x) sin(pi y) at every node."""
        f = (2 * np.pi ** 2 + lam) * np.sin(np.pi * self.x) * np.sin(np.pi * self.y)
        bL = (self.wJ[:, None] * f) @ self.MM.T
        return self.gather(bL.ravel())

    def jacobi_diag(self, lam=1.0):
        d = (self.ggeo[:, 0:1] * np.diag(self.Srr)[None, :] + self.ggeo[:, 1:2] * np.diag(self.Srs)[None, :]
             + self.ggeo[:, 2:3] * np.diag(self.Sss)[None, :] + lam * self.wJ[:, None] * np.diag(self.MM)[None, :])
        return self.gather(d.ravel())

    def cg(self, b, lam=1.0, tol=0.0, maxit=100, precon=False):
        """cg::Solve (libs/core/linearSolverCG.cpp:62-129) with optional Jacobi;
        returns (x, iterations, residual-norm history)."""
        x = np.zeros(self.Ngather)
        r = np.array(b, dtype=np.float64)
        invD = 1.0 / self.jacobi_diag(lam) if precon else None
        p = np.zeros_like(r)
        rdotr0 = r @ r
        hist = []
        rz_old = None
        it = 0
        for it in range(1, maxit + 1):
            z = invD * r if precon else r.copy()   # p must not alias r
            rz = r @ z
            p = z if rz_old is None else z + (rz / rz_old) * p
            rz_old = rz
            Ap = self.operator(p, lam)
            alpha = rz / (p @ Ap)
            x += alpha * p
            r -= alpha * Ap
            rdotr = r @ r
            hist.append(np.sqrt(rdotr))
            if rdotr <= tol * tol * rdotr0:
                break
        return x, it, np.array(hist)
