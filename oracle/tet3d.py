"""CPU restatement of the reference's Tet3D BP5 path (numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the library's
Tet3D meshes and operators; the product package never imports it.

What it restates (reference files, paths relative to the reference root):
  nodes        equispaced (r, s, t) layers (libs/mesh/meshBasisTet3D.cpp:227-248)
               warped and blended (Warburton 2006, :604-763): per face the 2D
               warp of WarpShiftFace3D along the face's two unit tangents,
               blended by Lb Lc Ld, with the face's own warp on its edges, then
               mapped back from the equilateral tetrahedron (:564-602)
  matrices     Dr, Ds, Dt = Vr,s,t V^-1, MM = (V V^T)^-1 of an orthonormal basis
               of P_N; the six stiffness matrices Srr, Srs (= Dr^T MM Ds +
               Ds^T MM Dr), Srt, Sss, Sst, Stt (:494-527)
  box          six tetrahedra per cell (meshSetupBoxTet3D.cpp), vertex
               orders as the reference writes them
  geometry     affine factors per element: J and
               G_ab = J (grad a . grad b), a, b in r, s, t
               (meshGeometricFactorsTet3D.cpp:31-110)
  numbering    as for Tri2D (oracle/tri2d.py): lowest copy, copy-wise masking
               on boundary faces, rows in first-unmasked-copy order
  operator     AqL_e = sum G_ab S_ab q_e + lambda J MM q_e
               (okl/bp5AxAffineTet3D.okl)

Parity pin: tests/golden/ref_tet_*.npz written by the reference's own set-up
code (tests/golden/make_golden.py), held by tests/test_tet3d.py.
"""
import numpy as np

from oracle import oracle as _o
from oracle import tri2d as _tri
from oracle.tri2d import _jacobi, _warp

ALPHA_OPT = [0.0000, 0.0000, 0.00000, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577, 1.1603, 1.10153, 0.6080, 0.4523,
             0.8856, 0.8717, 0.9655]

_V1 = np.array([-1.0, -1 / np.sqrt(3.0), -1 / np.sqrt(6.0)])
_V2 = np.array([1.0, -1 / np.sqrt(3.0), -1 / np.sqrt(6.0)])
_V3 = np.array([0.0, 2 / np.sqrt(3.0), -1 / np.sqrt(6.0)])
_V4 = np.array([0.0, 0.0, 3 / np.sqrt(6.0)])


def _face_warp(N, alpha, L1, L2, L3):
    """The 2D warp of a face (two tangential components)."""
    w1 = 4 * L2 * L3 * _warp(N, L3 - L2) * (1 + (alpha * L1) ** 2)
    w2 = 4 * L3 * L1 * _warp(N, L1 - L3) * (1 + (alpha * L2) ** 2)
    w3 = 4 * L1 * L2 * _warp(N, L2 - L1) * (1 + (alpha * L3) ** 2)
    return (w1 + np.cos(2 * np.pi / 3) * w2 + np.cos(4 * np.pi / 3) * w3,
            np.sin(2 * np.pi / 3) * w2 + np.sin(4 * np.pi / 3) * w3)


def nodes(N):
    """Warp & blend nodes (r, s, t) in the reference's order."""
    r, s, t = [], [], []
    for k in range(N + 1):
        for n in range(N + 1 - k):
            for m in range(N + 1 - n - k):
                r.append(-1.0 + 2.0 * m / N)
                s.append(-1.0 + 2.0 * n / N)
                t.append(-1.0 + 2.0 * k / N)
    r, s, t = np.array(r), np.array(s), np.array(t)
    alpha = ALPHA_OPT[N - 1] if N < 16 else 1.0
    t1 = [_V2 - _V1, _V2 - _V1, _V3 - _V2, _V3 - _V1]
    t2 = [_V3 - 0.5 * (_V1 + _V2), _V4 - 0.5 * (_V1 + _V2), _V4 - 0.5 * (_V2 + _V3), _V4 - 0.5 * (_V1 + _V3)]
    t1 = [v / np.linalg.norm(v) for v in t1]
    t2 = [v / np.linalg.norm(v) for v in t2]
    L1, L2, L3, L4 = 0.5 * (1 + t), 0.5 * (1 + s), -0.5 * (1 + r + s + t), 0.5 * (1 + r)
    X = np.outer(L3, _V1) + np.outer(L4, _V2) + np.outer(L2, _V3) + np.outer(L1, _V4)
    shift = np.zeros_like(X)
    faces = [(L1, L2, L3, L4), (L2, L1, L3, L4), (L3, L1, L4, L2), (L4, L1, L3, L2)]
    tol = 1e-10
    for f, (La, Lb, Lc, Ld) in enumerate(faces):
        w1, w2 = _face_warp(N, alpha, Lb, Lc, Ld)
        blend = Lb * Lc * Ld
        denom = (Lb + 0.5 * La) * (Lc + 0.5 * La) * (Ld + 0.5 * La)
        big = denom > tol
        blend = np.where(big, (1 + (alpha * La) ** 2) * blend / np.where(big, denom, 1.0), blend)
        shift += np.outer(blend * w1, t1[f]) + np.outer(blend * w2, t2[f])
        edge = (La < tol) & ((Lb < tol) | (Lc < tol) | (Ld < tol))
        shift[edge] = np.outer(w1[edge], t1[f]) + np.outer(w2[edge], t2[f])
    X = X + shift
    A = 0.5 * np.array([_V2 - _V1, _V3 - _V1, _V4 - _V1])
    B = X - 0.5 * (_V2 + _V3 + _V4 - _V1)
    RST = np.linalg.solve(A.T, B.T).T
    return RST[:, 0], RST[:, 1], RST[:, 2]


def vandermonde(N, r, s, t):
    """V, Vr, Vs, Vt of the orthonormal basis of P_N on the tetrahedron."""
    r, s, t = (np.asarray(v, dtype=np.float64) for v in (r, s, t))
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(np.abs(s + t) > 1e-14, 2 * (1 + r) / (-s - t) - 1, -1.0)
        b = np.where(np.abs(t - 1) > 1e-14, 2 * (1 + s) / (1 - t) - 1, -1.0)
    c = t
    V, Vr, Vs, Vt = [], [], [], []
    for i in range(N + 1):
        for j in range(N + 1 - i):
            for k in range(N + 1 - i - j):
                fa, dfa = _jacobi(a, 0, 0, i)
                gb, dgb = _jacobi(b, 2 * i + 1, 0, j)
                hc, dhc = _jacobi(c, 2 * (i + j) + 2, 0, k)
                V.append(2 * np.sqrt(2.0) * fa * gb * (1 - b) ** i * hc * (1 - c) ** (i + j))
                dr = dfa * gb * hc
                if i > 0:
                    dr = dr * (0.5 * (1 - b)) ** (i - 1)
                if i + j > 0:
                    dr = dr * (0.5 * (1 - c)) ** (i + j - 1)
                ds = 0.5 * (1 + a) * dr
                tmp = dgb * (0.5 * (1 - b)) ** i
                if i > 0:
                    tmp = tmp - 0.5 * i * gb * (0.5 * (1 - b)) ** (i - 1)
                if i + j > 0:
                    tmp = tmp * (0.5 * (1 - c)) ** (i + j - 1)
                tmp = fa * tmp * hc
                ds = ds + tmp
                dt = 0.5 * (1 + a) * dr + 0.5 * (1 + b) * tmp
                tmp = dhc * (0.5 * (1 - c)) ** (i + j)
                if i + j > 0:
                    tmp = tmp - 0.5 * (i + j) * hc * (0.5 * (1 - c)) ** (i + j - 1)
                tmp = fa * gb * tmp * (0.5 * (1 - b)) ** i
                dt = dt + tmp
                sc = 2 ** (2 * i + j + 1.5)
                Vr.append(dr * sc)
                Vs.append(ds * sc)
                Vt.append(dt * sc)
    return np.array(V).T, np.array(Vr).T, np.array(Vs).T, np.array(Vt).T


def reference_matrices(N):
    """r, s, t, Dr, Ds, Dt, MM, S (6 x Np x Np: rr, rs, rt, ss, st, tt), row-major."""
    r, s, t = nodes(N)
    V, Vr, Vs, Vt = vandermonde(N, r, s, t)
    Vi = np.linalg.inv(V)
    Dr, Ds, Dt = Vr @ Vi, Vs @ Vi, Vt @ Vi
    MM = np.linalg.inv(V @ V.T)
    D = (Dr, Ds, Dt)
    S = []
    for a, b in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)):
        X = D[a].T @ MM @ D[b]
        S.append(X if a == b else X + D[b].T @ MM @ D[a])
    return r, s, t, Dr, Ds, Dt, MM, np.array(S)


# cube corners (bit 0: x, bit 1: y, bit 2: z) of the six tetrahedra of a cell
TETS = [(0, 3, 2, 7), (0, 1, 3, 7), (0, 2, 6, 7), (0, 6, 4, 7), (0, 5, 1, 7), (0, 4, 5, 7)]


class Mesh:
    """The Tet3D box [-1,1]^3 of nx*ny*nz cells, six tetrahedra each, degree N."""

    def __init__(self, nx, ny, nz, N, tets=TETS):
        self.N = N
        self.Np = (N + 1) * (N + 2) * (N + 3) // 6
        self.E = 6 * nx * ny * nz
        (self.r, self.s, self.t, self.Dr, self.Ds, self.Dt, self.MM, self.S) = reference_matrices(N)
        dx, dy, dz = 2.0 / nx, 2.0 / ny, 2.0 / nz
        NnX, NnY = nx + 1, ny + 1
        EToV, EX, EY, EZ = [], [], [], []
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    x0, y0, z0 = -1.0 + dx * i, -1.0 + dy * j, -1.0 + dz * k
                    for tet in tets:
                        for c in tet:
                            ci, cj, ck = c & 1, (c >> 1) & 1, (c >> 2) & 1
                            EToV.append((i + ci) + (j + cj) * NnX + (k + ck) * NnX * NnY)
                            EX.append(x0 + dx if ci else x0)
                            EY.append(y0 + dy if cj else y0)
                            EZ.append(z0 + dz if ck else z0)
        self.EToV = np.array(EToV, np.int64)
        self.EX, self.EY, self.EZ = np.array(EX), np.array(EY), np.array(EZ)
        V = [a.reshape(-1, 4) for a in (self.EX, self.EY, self.EZ)]
        r, s, t = self.r, self.s, self.t
        w = [-(1 + r + s + t) / 2, (1 + r) / 2, (1 + s) / 2, (1 + t) / 2]
        self.x, self.y, self.z = (sum(np.outer(c[:, v], w[v]) for v in range(4)) for c in V)
        ex, ey, ez = V
        xr, xs, xt = [(c[:, v] - c[:, 0]) / 2 for c in (ex,) for v in (1, 2, 3)]
        yr, ys, yt = [(c[:, v] - c[:, 0]) / 2 for c in (ey,) for v in (1, 2, 3)]
        zr, zs, zt = [(c[:, v] - c[:, 0]) / 2 for c in (ez,) for v in (1, 2, 3)]
        J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt)
        rx, ry, rz = (ys * zt - zs * yt) / J, -(xs * zt - zs * xt) / J, (xs * yt - ys * xt) / J
        sx, sy, sz = -(yr * zt - zr * yt) / J, (xr * zt - zr * xt) / J, -(xr * yt - yr * xt) / J
        tx, ty, tz = (yr * zs - zr * ys) / J, -(xr * zs - zr * xs) / J, (xr * ys - yr * xs) / J
        self.wJ = J
        self.ggeo = np.stack([J * (rx * rx + ry * ry + rz * rz), J * (rx * sx + ry * sy + rz * sz),
                              J * (rx * tx + ry * ty + rz * tz), J * (sx * sx + sy * sy + sz * sz),
                              J * (sx * tx + sy * ty + sz * tz), J * (tx * tx + ty * ty + tz * tz)], axis=1)
        self._number()

    def _number(self):
        Np, E = self.Np, self.E
        key = np.round(np.stack([self.x.ravel(), self.y.ravel(), self.z.ravel()], axis=1) * 1e9).astype(np.int64)
        _, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.ravel()
        gmin = np.full(inv.max() + 1, np.iinfo(np.int64).max)
        np.minimum.at(gmin, inv, np.arange(E * Np) + 1)
        self.globalIds = gmin[inv]
        # faces 0..3 of the reference element: t = -1, s = -1, r + s + t = -1, r = -1
        tol = 1e-5
        r, s, t = self.r, self.s, self.t
        fnodes = [np.flatnonzero(np.abs(t + 1) < tol), np.flatnonzero(np.abs(s + 1) < tol),
                  np.flatnonzero(np.abs(r + s + t + 1) < tol), np.flatnonzero(np.abs(r + 1) < tol)]
        fverts = [(0, 1, 2), (0, 1, 3), (1, 2, 3), (0, 2, 3)]
        cs = [self.EX.reshape(-1, 4), self.EY.reshape(-1, 4), self.EZ.reshape(-1, 4)]
        masked = np.zeros(E * Np, bool)
        for e in range(E):
            for f, vs in enumerate(fverts):
                on = any(all(abs(c[e, v] - b) < 1e-12 for v in vs) for c in cs for b in (-1.0, 1.0))
                if on:
                    masked[e * Np + fnodes[f]] = True
        row = {}
        for l in np.flatnonzero(~masked):
            row.setdefault(self.globalIds[l], len(row))
        self.G2L = np.array([-1 if masked[l] else row[self.globalIds[l]] for l in range(E * Np)], np.int32)
        self.Ngather = len(row)
        cols = [[] for _ in range(self.Ngather)]
        for l in range(E * Np):
            if self.G2L[l] >= 0:
                cols[self.G2L[l]].append(l)
        self.rowStarts = np.zeros(self.Ngather + 1, np.int32)
        self.rowStarts[1:] = np.cumsum([len(c) for c in cols])
        self.colIds = np.array([c for cl in cols for c in cl], np.int32)

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
        qL = self.scatter(q).reshape(self.E, self.Np)
        out = np.zeros_like(qL)
        for a in range(6):
            out += self.ggeo[:, a:a + 1] * (qL @ self.S[a].T)
        out += lam * self.wJ[:, None] * (qL @ self.MM.T)
        return out.ravel()

    def operator(self, q, lam=1.0):
        return self.gather(self.ax(q, lam))

    def rhs_random(self, seed=0):
        f = 2.0 * _o.random(seed, self.Ngather) - 1.0
        fL = self.scatter(f).reshape(self.E, self.Np)
        return f, self.gather((self.wJ[:, None] * (fL @ self.MM.T)).ravel())

    def rhs_analytic(self, lam=1.0):
        """rhsAffineTet3D (okl/rhsTet3D.okl): Gather(MM (J f)) with
        f = (3 pi^2 + lambda) sin(pi x) sin(pi y) sin(pi z) at every node."""
        f = (3 * np.pi ** 2 + lam) * np.sin(np.pi * self.x) * np.sin(np.pi * self.y) * np.sin(np.pi * self.z)
        return self.gather(((self.wJ[:, None] * f) @ self.MM.T).ravel())

    cg = _tri.Mesh.cg   # cg::Solve with optional Jacobi, on this mesh's operator

    def jacobi_diag(self, lam=1.0):
        d = sum(self.ggeo[:, a:a + 1] * np.diag(self.S[a])[None, :] for a in range(6))
        d = d + lam * self.wJ[:, None] * np.diag(self.MM)[None, :]
        return self.gather(d.ravel())
