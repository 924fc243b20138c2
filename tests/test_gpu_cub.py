"""GPU parity of the over-integrated operators (BP1-BP4) against the oracle.

Same bars as the BP5/BP6 path: element operator, assembled operator and
diagonal within 1e-12 relative in FP64, cubature factors within 1e-13, CG
residual history within 1e-10 relative per iteration while the residual is
above 1e-6 of its start.
"""
import numpy as np
import pytest

from test_gpu_parity import HIST_TOL, _check_history, _rel

pytestmark = pytest.mark.gpu

AX_TOL = 1e-12

CUB_AX_CASES = ([(2, 2, 2, N, aff, 0.0 if aff else 0.1, bp) for N in (1, 2, 3, 4, 5, 6, 7, 8, 9, 11, 13, 15)
                 for aff in (False, True) for bp in (1, 3)] +
                [(2, 3, 2, N, aff, 0.0 if aff else 0.1, bp) for N in (1, 4, 7, 10, 15) for aff in (False, True)
                 for bp in (2, 4)] + [(3, 2, 2, 7, False, 0.2, 3), (4, 3, 2, 5, False, 0.1, 1)])


@pytest.mark.parametrize("nx,ny,nz,N,affine,pert,bpn", CUB_AX_CASES)
def test_cub_ax_matches_oracle(gpu, oracle, nx, ny, nz, N, affine, pert, bpn):
    Nf = 1 if bpn % 2 else 3
    om = oracle.Mesh(nx, ny, nz, N, affine=affine, Nfields=Nf, pert=pert)
    gm = gpu.Mesh(nx, ny, nz, N=N, affine=affine, Nfields=Nf, pert=pert)
    # cubature data set up on the device against the oracle's restatement
    for name, tol in (("cubr", 1e-15), ("cubw", 1e-14), ("cubInterp", 1e-13), ("cubD", 1e-13)):
        assert _rel(gm.array(name), om.array(name)) < tol, name
    if affine:
        assert _rel(gm.array("invV"), om.array("invV")) < 1e-13
    else:
        assert _rel(gm.array("cubwJ"), om.array("cubwJ")) < 1e-13
        assert _rel(gm.array("cubggeo"), om.array("cubggeo")) < 1e-13
    if om.Ngather == 0:
        return
    q = 2 * oracle.random(5, om.Ngather) - 1
    dq, dAq = gpu.DeviceBuffer.from_host(q), gpu.DeviceBuffer(om.NL)
    gpu.ax_cub_hex3d(gm, bpn, dq, dAq, lam=1.0)
    assert _rel(dAq.download(), om.ax(q, 1.0, bpn)) < AX_TOL


@pytest.mark.parametrize("bpn,affine,pert", [(1, False, 0.1), (1, True, 0.0), (2, False, 0.1), (3, False, 0.1),
                                            (3, True, 0.0), (4, False, 0.0), (4, True, 0.0)])
def test_cub_operator_forcing_and_diagonal(gpu, oracle, bpn, affine, pert):
    Nf = 1 if bpn % 2 else 3
    om = oracle.Mesh(3, 3, 2, 4, affine=affine, Nfields=Nf, pert=pert)
    gm = gpu.Mesh(3, 3, 2, N=4, affine=affine, Nfields=Nf, pert=pert)
    S = gpu.BP(gm, bp=bpn)
    q = 2 * oracle.random(3, om.Ngather) - 1
    dq, dAq = gpu.DeviceBuffer.from_host(q), gpu.DeviceBuffer(om.Ngather)
    S.operator(dq, dAq)
    assert _rel(dAq.download(), om.operator(q, 1.0, bpn)) < AX_TOL
    # BP1/BP2 force with lambda = 0 (BP/BP1/src/bp1Run.cpp:54-62)
    lam_rhs = 0.0 if bpn <= 2 else 1.0
    assert _rel(S.rhs("ANALYTIC").download(), om.rhs_analytic(lam_rhs)) < 1e-12
    assert _rel(S.diagonal().download(), om.jacobi_diag(1.0, bpn)) < 1e-12


CUB_CG_CASES = [(3, 6, 6, 6, 5, False, 0.1, "NONE"), (3, 6, 6, 6, 5, False, 0.1, "JACOBI"),
                (3, 8, 8, 8, 3, True, 0.0, "NONE"), (3, 3, 3, 3, 9, False, 0.1, "JACOBI"),
                (1, 6, 6, 6, 5, False, 0.1, "NONE"), (1, 5, 5, 5, 4, True, 0.0, "JACOBI"),
                (4, 4, 4, 4, 4, False, 0.1, "JACOBI"), (2, 4, 4, 4, 3, False, 0.1, "NONE")]


@pytest.mark.parametrize("bpn,nx,ny,nz,N,affine,pert,precon", CUB_CG_CASES)
def test_cub_cg_history_matches_oracle(gpu, oracle, bpn, nx, ny, nz, N, affine, pert, precon):
    Nf = 1 if bpn % 2 else 3
    om = oracle.Mesh(nx, ny, nz, N, affine=affine, Nfields=Nf, pert=pert)
    gm = gpu.Mesh(nx, ny, nz, N=N, affine=affine, Nfields=Nf, pert=pert)
    S = gpu.BP(gm, bp=bpn, precon=precon)
    b_o = om.rhs_random(0)[1]
    maxit = 60
    x_o, r_o, it_o, hr_o, ha_o = om.cg(b_o, 1.0, 0.0, maxit, precon=(precon == "JACOBI"), bp=bpn)
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    st, hr, ha = S.solve(x, S.rhs("RANDOM", 0), tol=0.0, maxit=maxit)
    assert st.iterations == it_o == maxit
    # How far this problem's history is reproducible at all: the oracle run
    # again on b perturbed by 1e-15 relative (a rounding-sized change), four
    # draws, the worst of them.  The mass matrices cluster their spectrum and
    # amplify such a change fast (measured on BP1 5^3 p=4 with Jacobi: the
    # four draws differ from the unperturbed run by 3e-12 to 2e-10 at
    # iteration 12, r/r0 = 1.5e-5, and one draw alone can miss that; the
    # oracle's own affine and curved operators 1e-15 apart give the same).
    # The 1e-10 bar holds up to the first iteration where the oracle
    # disagrees with itself by more than 1e-11.
    self_rel = np.zeros(maxit)
    for seed in (99, 98, 97, 96):
        noise = 1.0 + 1e-15 * (2 * oracle.random(seed, om.Ngather) - 1)
        _, _, _, hr_p, _ = om.cg(b_o * noise, 1.0, 0.0, maxit, precon=(precon == "JACOBI"), bp=bpn)
        self_rel = np.maximum(self_rel, np.abs(hr_p - hr_o) / hr_o)
    bad = np.flatnonzero(self_rel > HIST_TOL / 10)
    reproducible = np.arange(maxit) < (bad[0] if bad.size else maxit)
    live = _check_history(hr[reproducible], hr_o[reproducible])
    assert np.all((np.abs(ha - ha_o) / np.abs(ha_o))[reproducible][live] < HIST_TOL)
    # past that range: as converged as the oracle, and the same solution
    assert hr[-1] <= max(100 * hr_o[-1], 1e-12 * hr_o[0])
    assert _rel(x.download(), x_o) < 1e-9


@pytest.mark.parametrize("bpn,affine,pert", [(3, False, 0.1), (1, False, 0.1), (4, True, 0.0)])
def test_cub_mixed_precision_reaches_tolerance(gpu, oracle, bpn, affine, pert):
    Nf = 1 if bpn % 2 else 3
    om = oracle.Mesh(5, 5, 5, 5, affine=affine, Nfields=Nf, pert=pert)
    gm = gpu.Mesh(5, 5, 5, N=5, affine=affine, Nfields=Nf, pert=pert)
    S = gpu.BP(gm, bp=bpn, precon="JACOBI", precision="MIXED")
    b_o = om.rhs_random(0)[1]
    x_o, _, it_o, _, _ = om.cg(b_o, 1.0, 1e-8, 5000, precon=True, bp=bpn)
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    st, _, _ = S.solve(x, gpu.DeviceBuffer.from_host(b_o), tol=1e-8, maxit=5000)
    assert st.iterations <= 1.25 * it_o + 20
    xs = x.download()
    # FP64 residual of the returned solution, by the oracle operator
    r = b_o - om.operator(xs, 1.0, bpn)
    assert np.linalg.norm(r) <= 1.0001e-8 * np.linalg.norm(b_o)
    assert _rel(xs, x_o) < 1e-5


def test_cub_bad_arguments_fail_loudly(gpu):
    gm = gpu.Mesh(2, 2, 2, N=3)
    with pytest.raises(gpu.BPError):
        gpu.BP(gm, bp=4)                  # BP4 needs three fields
    dq, dAq = gpu.DeviceBuffer(gm.Ngather), gpu.DeviceBuffer(gm.NL)
    with pytest.raises(gpu.BPError):
        gpu.ax_cub_hex3d(gm, 5, dq, dAq)  # the cubature kernel covers BP1-BP4 only


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_cub_driver_result_lines(gpu, capfd, k):
    assert gpu.driver_main("BP%d" % k, ["-nx", "3", "-ny", "3", "-nz", "3", "-p", "4", "-wi", "5", "-it", "20"]) == 0
    out = capfd.readouterr().out
    line = [l for l in out.splitlines() if l.startswith("BP%d: N=" % k)][0]
    assert "iterations=20, time per DOF=" in line and line.endswith("Element=Hex ")
    assert gpu.driver_main("BK%d" % k, ["-nx", "3", "-ny", "3", "-nz", "3", "-p", "4", "-a"]) == 0
    out = capfd.readouterr().out
    assert [l for l in out.splitlines() if l.startswith("BK%d: N= 4," % k)][0].endswith("Element=Hex, Affine ")


@pytest.mark.parametrize("bpn,N,affine", [(3, 7, False), (3, 4, False), (1, 7, False), (4, 5, False), (3, 6, True),
                                          (1, 5, True)])
def test_cub_fp32_operator_matches_oracle(gpu, oracle, bpn, N, affine):
    # the FP32 over-integrated operator (the mixed-precision solver's inner
    # operator) is the FP64 oracle's to FP32 accuracy
    Nf = 1 if bpn % 2 else 3
    pert = 0.0 if affine else 0.1
    om = oracle.Mesh(3, 2, 2, N, affine=affine, Nfields=Nf, pert=pert)
    gm = gpu.Mesh(3, 2, 2, N=N, affine=affine, Nfields=Nf, pert=pert)
    c = gm.cubature()
    G, Nq = c.cubNq, gm.Nq
    nc = gm.E if affine else gm.E * c.cubNp
    sizes = {"cubwJ": nc, "cubggeo": 6 * nc, "cubD": Nq * Nq if affine else G * G, "cubInterp": G * Nq,
             "invV": Nq * Nq, "MM": Nq * Nq}
    f32 = {}
    for name, n in sizes.items():
        f32[name] = gpu.DeviceBuffer(n, np.float32)
        gpu.convert_f64_f32(getattr(c, name), n, f32[name])
    q = 2 * oracle.random(8, om.Ngather) - 1
    dq = gpu.DeviceBuffer.from_host(q.astype(np.float32))
    dA = gpu.DeviceBuffer(om.NL, np.float32)
    d = gpu.AxDesc(bpn, N, int(affine), Nf)
    v = gm.view
    gpu._check(gpu.lib().bp_ax_cub_hex3d_f32(gpu.ctypes.byref(d), gm.E, v.elementList, v.GlobalToLocal,
                                             f32["cubwJ"].ptr, f32["cubggeo"].ptr, f32["cubD"].ptr,
                                             f32["cubInterp"].ptr, f32["invV"].ptr, f32["MM"].ptr, 1.0, dq.ptr,
                                             dA.ptr, None))
    want = om.ax(q.astype(np.float32).astype(np.float64), 1.0, bpn)
    assert _rel(dA.download().astype(np.float64), want) < 2e-5
