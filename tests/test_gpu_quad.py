"""Quad2D (the reference's 2D tensor-product element) through the C ABI: the
device mesh, the BP5/BP6 element operators (FP64 and FP32), forcing, Jacobi
diagonal and CG against the oracle's restatement of okl/bp5AxQuad2D.okl,
okl/bp5AxAffineQuad2D.okl, okl/bp6AxQuad2D.okl and okl/rhsQuad2D.okl (itself
held to the reference's own Quad2D set-up by tests/test_ref_golden.py).

Bars as for Hex3D: indexing bit-exact; FP64 operator, forcing and diagonal
within 1e-12 relative; gather bit-exact on the same E-vector; CG residual
history within 1e-10 relative per iteration while the residual is above 1e-6
r0; the FP32 operator within 2e-6 of the FP64 oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AX_TOL = 1e-12
HIST_TOL = 1e-10


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


CASES = [(4, 3, N, False, 0.1, 1) for N in (1, 2, 3, 4, 5, 6, 7, 8, 11, 15)] + [
    (5, 4, 7, True, 0.0, 1), (3, 3, 15, True, 0.0, 1), (4, 3, 5, False, 0.2, 2), (3, 4, 4, True, 0.0, 2),
    (1, 1, 1, False, 0.0, 1), (6, 2, 9, False, 0.1, 2)]


@pytest.mark.parametrize("nx,ny,N,affine,pert,nf", CASES)
def test_quad_mesh_operator_gather_match_oracle(gpu, oracle, nx, ny, N, affine, pert, nf):
    om = oracle.Mesh(nx, ny, 0, N, affine=affine, Nfields=nf, pert=pert, dim=2)
    gm = gpu.Mesh(nx, ny, N=N, affine=affine, Nfields=nf, pert=pert, dim=2)
    assert gm.dim == 2 and (gm.Np, gm.Ngather, gm.nnz) == (om.Np, om.Ngather, om.nnz)
    np.testing.assert_array_equal(gm.array("GlobalToLocal"), om.array("G2L"))
    np.testing.assert_array_equal(gm.array("rowStarts"), om.array("rowStarts"))
    np.testing.assert_array_equal(gm.array("colIds"), om.array("colIds"))
    np.testing.assert_array_equal(gm.array("EX"), om.array("EX"))
    np.testing.assert_array_equal(gm.array("EY"), om.array("EY"))
    assert _rel(gm.array("wJ"), om.array("wJ")) < 1e-13
    assert _rel(gm.array("ggeo"), om.array("ggeo")) < 1e-13
    if om.Ngather == 0:
        return
    q = 2 * oracle.random(13, om.Ngather) - 1
    dq, dA = gpu.DeviceBuffer.from_host(q), gpu.DeviceBuffer(om.NL)
    gpu.ax_hex3d(gm, dq, dA)
    AqL = dA.download()
    assert _rel(AqL, om.ax(q)) < AX_TOL
    dg = gpu.DeviceBuffer(om.Ngather)
    gpu.ogs_gather(gm, dA, dg)
    np.testing.assert_array_equal(dg.download(), om.gather(AqL))
    # the FP32 operator (the mixed-precision solver's inner operator)
    v = gm.view
    ng = gm.E if gm.affine else gm.E * gm.Np
    ops = {"wJ": gpu.DeviceBuffer(ng, np.float32), "ggeo": gpu.DeviceBuffer(3 * ng, np.float32),
           "gllw": gpu.DeviceBuffer(gm.Nq, np.float32), "D": gpu.DeviceBuffer(gm.Nq * gm.Nq, np.float32)}
    for name, n in (("wJ", ng), ("ggeo", 3 * ng), ("gllw", gm.Nq), ("D", gm.Nq * gm.Nq)):
        gpu.convert_f64_f32(getattr(v, name), n, ops[name])
    q32 = gpu.DeviceBuffer.from_host(q.astype(np.float32))
    A32 = gpu.DeviceBuffer(om.NL, np.float32)
    gpu.ax_hex3d_f32(gm, q32, A32, ops)
    assert _rel(A32.download().astype(np.float64), om.ax(q.astype(np.float32).astype(np.float64))) < 2e-6


@pytest.mark.parametrize("nx,ny,N,affine,pert,nf", [(4, 3, 5, False, 0.1, 1), (3, 3, 7, True, 0.0, 1),
                                                    (4, 4, 4, False, 0.1, 2)])
def test_quad_forcing_and_diagonal_match_oracle(gpu, oracle, nx, ny, N, affine, pert, nf):
    om = oracle.Mesh(nx, ny, 0, N, affine=affine, Nfields=nf, pert=pert, dim=2)
    gm = gpu.Mesh(nx, ny, N=N, affine=affine, Nfields=nf, pert=pert, dim=2)
    S = gpu.BP(gm, precon="JACOBI")
    assert _rel(S.rhs("ANALYTIC").download(), om.rhs_analytic(1.0)) < 1e-13
    f = gpu.DeviceBuffer(om.Ngather)
    b = S.rhs("RANDOM", 3, f=f)
    f_o, b_o = om.rhs_random(3)
    np.testing.assert_array_equal(f.download(), f_o)
    assert _rel(b.download(), b_o) < 1e-13
    d = gpu.DeviceBuffer(om.Ngather)
    gpu._check(gpu.lib().bp_solver_diagonal(S._h, d.ptr))
    assert _rel(d.download(), om.jacobi_diag(1.0)) < AX_TOL


@pytest.mark.parametrize("nx,ny,N,affine,pert,nf,precon", [(6, 5, 5, False, 0.1, 1, "JACOBI"),
                                                           (8, 8, 3, True, 0.0, 1, "NONE"),
                                                           (5, 4, 7, False, 0.1, 2, "JACOBI")])
def test_quad_cg_history_matches_oracle(gpu, oracle, nx, ny, N, affine, pert, nf, precon):
    om = oracle.Mesh(nx, ny, 0, N, affine=affine, Nfields=nf, pert=pert, dim=2)
    gm = gpu.Mesh(nx, ny, N=N, affine=affine, Nfields=nf, pert=pert, dim=2)
    S = gpu.BP(gm, precon=precon)
    _, b_o = om.rhs_random(0)
    x_o, _, it_o, hr_o, ha_o = om.cg(b_o, 1.0, 0.0, 80, precon=(precon == "JACOBI"))
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    st, hr, ha = S.solve(x, S.rhs("RANDOM", 0), tol=0.0, maxit=80)
    assert st.iterations == it_o == 80
    live = hr_o >= 1e-6 * hr_o[0]
    assert live[:10].all()
    assert np.max((np.abs(hr - hr_o) / hr_o)[live]) < HIST_TOL
    assert np.max((np.abs(ha - ha_o) / np.abs(ha_o))[live]) < HIST_TOL
    assert np.all(np.abs(hr - hr_o) <= HIST_TOL * hr_o[0])


# affine: the FP32 column form of the operator (one thread per column of nodes)
@pytest.mark.parametrize("nf,affine", [(1, False), (2, False), (1, True), (2, True)])
def test_quad_mixed_solve_reaches_tolerance(gpu, oracle, nf, affine):
    pert = 0.0 if affine else 0.1
    om = oracle.Mesh(12, 10, 0, 6, Nfields=nf, pert=pert, affine=affine, dim=2)
    gm = gpu.Mesh(12, 10, N=6, Nfields=nf, pert=pert, affine=affine, dim=2)
    S = gpu.BP(gm, precon="JACOBI", precision="MIXED")
    _, b_o = om.rhs_random(1)
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    st, _, _ = S.solve(x, gpu.DeviceBuffer.from_host(b_o), tol=1e-8, maxit=5000)
    assert st.updates >= 1
    xh = x.download()
    assert np.linalg.norm(b_o - om.operator(xh)) <= 1.0001e-8 * np.linalg.norm(b_o)
    x64, _, _, _, _ = om.cg(b_o, 1.0, 1e-12, 5000, precon=True)
    assert _rel(xh, x64) < 1e-6


def test_quad_driver_result_line(gpu, capfd):
    assert gpu.driver_main("BP5", ["-e", "Quad", "-nx", "8", "-ny", "6", "-p", "5", "-pc", "JACOBI", "-wi", "5",
                                   "-it", "50"]) == 0
    out = capfd.readouterr().out
    line = [l for l in out.splitlines() if l.startswith("BP5: N=")][0]
    assert line.startswith("BP5: N= 5, DOFs=%d," % ((8 * 5 - 1) * (6 * 5 - 1)))
    assert "iterations=50," in line and line.rstrip().endswith("Element=Quad")
    assert gpu.driver_main("BK6", ["-e", "Quad", "-nx", "8", "-ny", "6", "-p", "7", "-a"]) == 0
    out = capfd.readouterr().out
    assert any(l.startswith("BK6: N= 7,") and "Element=Quad, Affine" in l for l in out.splitlines())


def test_quad_rejections(gpu):
    gm = gpu.Mesh(3, 3, N=4, dim=2)
    with pytest.raises(gpu.BPError):
        gpu.BP(gm, bp=3)                  # over-integrated forms are Hex3D only
    with pytest.raises(gpu.BPError):
        gpu.BP(gm, bp=6)                  # BP6 needs a 2-field Quad2D mesh
    with pytest.raises(gpu.BPError):
        gpu.Mesh(3, 3, N=4, Nfields=3, dim=2)
    assert gpu.driver_main("BP3", ["-e", "Quad", "-nx", "4", "-ny", "4"]) != 0
