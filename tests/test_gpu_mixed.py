"""Mixed-precision CG (FP32 recursion and operator, FP64 reliable updates).

The stop rule is on the FP64 residual, ||b - A x|| <= tol ||b||, so the
solution must satisfy it when re-checked with the FP64 operator, and agree
with the oracle's FP64 CG solution to the accuracy the tolerance implies.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(6, 6, 6, 7, False, 0.1, "JACOBI", 1), (8, 8, 8, 4, True, 0.0, "JACOBI", 1),
         (5, 5, 5, 5, False, 0.1, "NONE", 1), (4, 4, 4, 6, False, 0.1, "JACOBI", 3),
         (3, 3, 3, 9, False, 0.1, "JACOBI", 1)]


@pytest.mark.parametrize("nx,ny,nz,N,affine,pert,precon,Nf", CASES)
def test_mixed_reaches_fp64_tolerance(gpu, oracle, nx, ny, nz, N, affine, pert, precon, Nf):
    tol = 1e-8
    om = oracle.Mesh(nx, ny, nz, N, affine=affine, pert=pert, Nfields=Nf)
    gm = gpu.Mesh(nx, ny, nz, N=N, affine=affine, pert=pert, Nfields=Nf)
    Sm = gpu.BP(gm, precon=precon, precision="MIXED")
    S64 = gpu.BP(gm, precon=precon)
    _, b_o = om.rhs_random(0)
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    r = gpu.DeviceBuffer.from_host(b_o)
    st, hr, ha = Sm.solve(x, r, tol=tol, maxit=20000)
    assert st.updates >= 1
    xh = x.download()
    # independent FP64 check of the residual
    Ax = gpu.DeviceBuffer(om.Ngather)
    S64.operator(x, Ax)
    res = np.linalg.norm(b_o - Ax.download()) / np.linalg.norm(b_o)
    assert res <= tol * 1.0001, res
    assert abs(np.sqrt(st.rdotr / st.rdotr0) - res) <= 1e-3 * res + 1e-16
    # the FP64 oracle's CG to the same tolerance
    x_o, _, it_o, _, _ = om.cg(b_o, 1.0, tol, 20000, precon=(precon == "JACOBI"))
    err = np.linalg.norm(xh - x_o) / np.linalg.norm(x_o)
    assert err < 1e-5, err
    # the reliable updates keep the Krylov space: about FP64 CG's iteration count
    assert st.iterations <= 1.25 * it_o + 20, (st.iterations, it_o)


def test_mixed_needs_tolerance_and_reports_maxit(gpu):
    gm = gpu.Mesh(3, 3, 3, N=4)
    S = gpu.BP(gm, precon="JACOBI", precision="MIXED")
    b = S.rhs("RANDOM", 0)
    with pytest.raises(gpu.BPError, match="tol"):
        S.solve(gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather)), b, tol=0.0, maxit=10)
    b = S.rhs("RANDOM", 0)
    st, _, _ = S.solve(gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather)), b, tol=1e-14, maxit=7)
    assert st.iterations == 7


def test_mixed_host_entry_matches_device_entry(gpu):
    gm = gpu.Mesh(4, 4, 4, N=5, pert=0.1)
    S = gpu.BP(gm, precon="JACOBI", precision="MIXED")
    b = S.rhs("RANDOM", 0)
    bh = b.download()
    x = gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather))
    st, _, _ = S.solve(x, gpu.DeviceBuffer.from_host(bh), tol=1e-8, maxit=5000)
    xh = np.zeros(gm.Ngather)
    st2 = S.solve_host(bh, xh, tol=1e-8, maxit=5000)
    assert st2.iterations == st.iterations and st2.updates == st.updates
    np.testing.assert_array_equal(xh, x.download())


@pytest.mark.parametrize("N,nrhs", [(7, 4), (7, 2), (4, 4), (6, 2), (9, 2), (3, 4), (8, 4), (9, 4), (10, 4),
                                    (11, 4), (5, 4)])
def test_fp32_multi_rhs_operator_matches_single(gpu, oracle, N, nrhs):
    # the packed operator (TMA form at even Nq >= 8, line form otherwise) gives each
    # right-hand side what the single-rhs FP32 operator gives it, and both are
    # the FP64 oracle's operator to FP32 accuracy
    om = oracle.Mesh(3, 2, 2, N, pert=0.1)
    gm = gpu.Mesh(3, 2, 2, N=N, pert=0.1)
    v = gm.view
    ng = gm.E * gm.Np
    ops = {"wJ": gpu.DeviceBuffer(ng, np.float32), "ggeo": gpu.DeviceBuffer(6 * ng, np.float32),
           "gllw": gpu.DeviceBuffer(gm.Nq, np.float32), "D": gpu.DeviceBuffer(gm.Nq * gm.Nq, np.float32)}
    for name, n in (("wJ", ng), ("ggeo", 6 * ng), ("gllw", gm.Nq), ("D", gm.Nq * gm.Nq)):
        gpu.convert_f64_f32(getattr(v, name), n, ops[name])
    Q = np.stack([2 * oracle.random(20 + k, gm.Ngather) - 1 for k in range(nrhs)], axis=1).astype(np.float32)
    dq = gpu.DeviceBuffer.from_host(np.ascontiguousarray(Q).ravel())
    dA = gpu.DeviceBuffer(gm.NL * nrhs, np.float32)
    gpu.ax_hex3d_f32_multi(gm, nrhs, dq, dA, ops)
    A = dA.download().reshape(gm.NL, nrhs)
    for k in range(nrhs):
        q1 = gpu.DeviceBuffer.from_host(np.ascontiguousarray(Q[:, k]))
        a1 = gpu.DeviceBuffer(gm.NL, np.float32)
        gpu.ax_hex3d_f32(gm, q1, a1, ops)
        single = a1.download()
        assert np.max(np.abs(A[:, k] - single)) <= 1e-6 * np.max(np.abs(single))
        want = om.ax(Q[:, k].astype(np.float64))
        assert np.max(np.abs(A[:, k] - want)) <= 2e-5 * np.max(np.abs(want))
