"""Tet3D (affine tetrahedra, BP5) through the C ABI: the device mesh against the
reference's own set-up (tests/golden/ref_tet_*.npz), bp_ax_tet3d, the gather,
the forcings, the Jacobi diagonal, FP64 and mixed-precision CG against the
oracle's restatement of okl/bp5AxAffineTet3D.okl (oracle/tet3d.py, itself held
to the same fixtures by tests/test_tet3d.py).

Bars as for the other elements: indexing bit-exact; operator, forcing and
diagonal within 1e-12 relative; CG residual history within 1e-10 relative per
iteration while the residual is above 1e-6 r0.
"""
import numpy as np
import pytest

from test_ref_golden import rel
from test_tet3d import SMALL, case, ids, mtol

pytestmark = pytest.mark.gpu

AX_TOL = 1e-12
HIST_TOL = 1e-10


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _tol(gpu, tet, N, base):
    """base, or above degree 9 four times the relative difference between the
    library's MM and S and the oracle's: both invert V V^T (the reference's
    MassMatrixTet3D), whose condition grows with N (1.5e-12 apart at N = 12,
    1e-10 at N = 15), and the rounding of the Np-long sums grows with Np."""
    if N <= 9:
        return base
    h, o = gpu.basis_tet3d(N), tet.reference_matrices(N)
    d = max(_rel(h[6], o[6]), _rel(h[7], o[7]))
    Np = (N + 1) * (N + 2) * (N + 3) // 6
    return max(base * Np / 220, 4 * d)


@pytest.fixture(scope="module")
def tet():
    from oracle import tet3d
    return tet3d


def _mesh(gpu, nx, ny, nz, N):
    return gpu.Mesh(nx, ny, nz, N=N, affine=True, dim=3, simplex=True)


@pytest.mark.parametrize("path", SMALL, ids=ids(SMALL))
def test_device_mesh_matches_reference_code(gpu, path):
    g, nx, ny, nz, N = case(path)
    m = _mesh(gpu, nx, ny, nz, N)
    Np = m.Np
    assert m.simplex and m.dim == 3 and (m.E, Np, m.Ngather) == (int(g["Nelements"][0]), int(g["Np"][0]),
                                                                  int(g["Ngather"][0]))
    np.testing.assert_array_equal(m.array("GlobalToLocal"), g["GlobalToLocal"])
    np.testing.assert_array_equal(m.array("rowStarts"), g["rowStartsT"])
    np.testing.assert_array_equal(m.array("colIds"), g["colIdsT"])
    for k in ("EX", "EY", "EZ"):
        assert rel(m.array(k), g[k]) <= 1e-15, k
    assert rel(m.array("wJ"), g["wJ"]) <= 1e-14 and rel(m.array("ggeo"), g["ggeo"]) <= 1e-14
    D = m.array("D").reshape(3, Np, Np).transpose(0, 2, 1)
    assert rel(D, g["D"].reshape(3, Np, Np)) <= mtol(N, Np)
    S = m.array("S").reshape(6, Np, Np).transpose(0, 2, 1)
    assert rel(S, g["S"].reshape(6, Np, Np)) <= mtol(N, Np)
    assert rel(m.array("MM"), g["MM"]) <= mtol(N, Np)
    gv = gpu.DeviceBuffer(m.Ngather)
    gpu.ogs_gather(m, gpu.DeviceBuffer.from_host(g["gather_in"]), gv)
    np.testing.assert_array_equal(gv.download(), g["gather_out"])


# degrees 12 and 15 have more nodes per element (455, 816) than the kernels'
# blocks have threads: their threads walk the nodes in strides
@pytest.mark.parametrize("nx,ny,nz,N", [(2, 2, 1, 3), (3, 2, 2, 4), (2, 2, 2, 7), (2, 1, 2, 1), (2, 2, 2, 9),
                                        (1, 1, 1, 2), (2, 1, 1, 12), (1, 1, 1, 15)])
def test_operator_matches_oracle(gpu, tet, nx, ny, nz, N):
    om = tet.Mesh(nx, ny, nz, N)
    gm = _mesh(gpu, nx, ny, nz, N)
    assert (gm.Ngather, gm.nnz) == (om.Ngather, om.colIds.size)
    if om.Ngather == 0:
        return
    q = 2 * np.random.default_rng(N).random(om.Ngather) - 1
    dq = gpu.DeviceBuffer.from_host(q)
    tol = _tol(gpu, tet, N, AX_TOL)
    for lam in (1.0, 0.0):
        dA = gpu.DeviceBuffer.from_host(np.full(om.NL, np.nan))
        gpu.ax_tet3d(gm, dq, dA, lam=lam)
        assert _rel(dA.download(), om.ax(q, lam)) < tol
    S = gpu.BP(gm, precon="NONE")
    Aq = gpu.DeviceBuffer(om.Ngather)
    S.operator(dq, Aq)
    assert _rel(Aq.download(), om.operator(q)) < tol


@pytest.mark.parametrize("nx,ny,nz,N", [(3, 2, 2, 5), (2, 1, 1, 12)])
def test_forcing_and_diagonal_match_oracle(gpu, tet, nx, ny, nz, N):
    om = tet.Mesh(nx, ny, nz, N)
    gm = _mesh(gpu, nx, ny, nz, N)
    S = gpu.BP(gm, precon="JACOBI")
    assert _rel(S.rhs("ANALYTIC").download(), om.rhs_analytic(1.0)) < _tol(gpu, tet, N, 1e-13)
    f = gpu.DeviceBuffer(om.Ngather)
    b = S.rhs("RANDOM", 3, f=f)
    f_o, b_o = om.rhs_random(3)
    np.testing.assert_array_equal(f.download(), f_o)
    assert _rel(b.download(), b_o) < _tol(gpu, tet, N, 1e-13)
    d = gpu.DeviceBuffer(om.Ngather)
    gpu._check(gpu.lib().bp_solver_diagonal(S._h, d.ptr))
    assert _rel(d.download(), om.jacobi_diag(1.0)) < _tol(gpu, tet, N, AX_TOL)


@pytest.mark.parametrize("nx,ny,nz,N,precon", [(3, 3, 2, 4, "JACOBI"), (3, 3, 3, 4, "NONE")])
def test_cg_history_matches_oracle(gpu, tet, nx, ny, nz, N, precon):
    om = tet.Mesh(nx, ny, nz, N)
    gm = _mesh(gpu, nx, ny, nz, N)
    S = gpu.BP(gm, precon=precon)
    _, b_o = om.rhs_random(0)
    _, it_o, hr_o = om.cg(b_o, 1.0, 0.0, 40, precon=(precon == "JACOBI"))
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    st, hr, _ = S.solve(x, S.rhs("RANDOM", 0), tol=0.0, maxit=40)
    assert st.iterations == it_o == 40
    live = hr_o >= 1e-6 * hr_o[0]
    assert live[:10].all()
    assert np.max((np.abs(hr - hr_o) / hr_o)[live]) < HIST_TOL
    assert np.all(np.abs(hr - hr_o) <= HIST_TOL * hr_o[0])


def test_mixed_solve_reaches_tolerance(gpu, tet):
    om = tet.Mesh(4, 3, 3, 4)
    gm = _mesh(gpu, 4, 3, 3, 4)
    S = gpu.BP(gm, precon="JACOBI", precision="MIXED")
    _, b_o = om.rhs_random(1)
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    st, _, _ = S.solve(x, gpu.DeviceBuffer.from_host(b_o), tol=1e-8, maxit=5000)
    assert st.updates >= 1
    xh = x.download()
    assert np.linalg.norm(b_o - om.operator(xh)) <= 1.0001e-8 * np.linalg.norm(b_o)


def test_driver_result_line_and_rejections(gpu, capfd):
    assert gpu.driver_main("BP5", ["-e", "Tet", "-nx", "4", "-ny", "4", "-nz", "3", "-p", "4", "-a", "-pc", "JACOBI",
                                   "-wi", "5", "-it", "30"]) == 0
    out = capfd.readouterr().out
    line = [l for l in out.splitlines() if l.startswith("BP5: N=")][0]
    assert "iterations=30," in line and line.rstrip().endswith("Element=Tet, Affine")
    assert gpu.driver_main("BK5", ["-e", "Tet", "-nx", "4", "-ny", "4", "-nz", "4", "-p", "5", "-a"]) == 0
    out = capfd.readouterr().out
    assert any(l.startswith("BK5: N= 5,") and "Element=Tet, Affine" in l for l in out.splitlines())
    assert gpu.driver_main("BP5", ["-e", "Tet", "-nx", "4", "-ny", "4", "-nz", "4"]) != 0   # needs -a
    gm = _mesh(gpu, 2, 2, 2, 3)
    with pytest.raises(gpu.BPError):
        gpu.BP(gm, bp=3)
