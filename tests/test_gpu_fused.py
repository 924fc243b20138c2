"""The CG direction update fused into the stored-factor element operator.

bp_cg_direction_ax_hex3d / bp_cg_direction_ax_f32_multi form p_new = invD r +
beta p_old, apply x += alpha p_old at the nodes they own and return A_e p_new,
in one pass over the factors.  Checked against the same steps done one by one:
numpy for the vector update (a few ulps: the kernel may contract z + beta p
into one fused multiply-add), the oracle's element operator (FP64, 1e-12) or
the unfused FP32 operator in the same form on the same p_new (bit for bit:
the same arithmetic on the same values), and the block partials of p.Ap
against p_new.A_e p_new.
Then whole CG solves with the fused and the unfused iteration side by side.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AX_TOL = 1e-12
HIST_TOL = 1e-10


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _owner(gpu, gm):
    om = gpu.DeviceBuffer(gm.NL, np.int32)
    gpu.ogs_owner_map(gm, om)
    return om


def test_owner_map_marks_first_column_of_every_row(gpu):
    gm = gpu.Mesh(3, 2, 2, N=4, pert=0.1)
    own = _owner(gpu, gm).download()
    g2l = gm.array("GlobalToLocal")
    rs, ci = gm.array("rowStarts"), gm.array("colIds")
    marked = own >= 0
    assert np.array_equal(own < 0, g2l < 0)
    assert np.array_equal(own[marked] & (gpu.OWNER_BIT - 1), g2l[marked])
    owners = np.flatnonzero((own >= 0) & ((own & gpu.OWNER_BIT) != 0))
    assert np.array_equal(np.sort(owners), np.sort(ci[rs[:-1]]))   # one owner per row, its first column


@pytest.mark.parametrize("nx,ny,nz,N,Nf,precon", [(3, 2, 2, 7, 1, True), (2, 3, 2, 5, 1, False),
                                                   (2, 2, 2, 3, 3, True), (1, 1, 1, 1, 1, True),
                                                   (2, 2, 2, 15, 1, True)])
def test_fused_step_fp64_matches_separate_steps(gpu, oracle, nx, ny, nz, N, Nf, precon):
    om = oracle.Mesh(nx, ny, nz, N, Nfields=Nf, pert=0.1)
    gm = gpu.Mesh(nx, ny, nz, N=N, Nfields=Nf, pert=0.1)
    Ng = om.Ngather
    own = _owner(gpu, gm)
    r = 2 * oracle.random(21, Ng) - 1
    pold = 2 * oracle.random(22, Ng) - 1
    x = 2 * oracle.random(23, Ng) - 1
    invD = 0.5 + oracle.random(24, Ng) if precon else None
    alpha, beta = 0.37, 0.81
    d = {k: gpu.DeviceBuffer.from_host(v) for k, v in (("r", r), ("p", pold), ("x", x))}
    dinv = gpu.DeviceBuffer.from_host(invD) if precon else None
    pnew = gpu.DeviceBuffer.from_host(np.full(Ng, np.nan))
    Aq = gpu.DeviceBuffer(om.NL)
    parts = gpu.DeviceBuffer.from_host(np.zeros(gm.E + 1))
    gpu.cg_direction_ax(gm, own, alpha, beta, d["r"], dinv, d["p"], pnew, d["x"], Aq, parts)
    if Ng == 0:   # every node masked: no vector is touched, A_e of the zero pencil
        assert not np.any(Aq.download())
        return
    z = (invD * r) if precon else r
    want_p = z + beta * pold
    got_p = pnew.download()
    assert _rel(got_p, want_p) < 4e-16
    assert _rel(d["x"].download(), x + alpha * pold) < 4e-16
    assert np.array_equal(d["p"].download(), pold) and np.array_equal(d["r"].download(), r)
    AqL = Aq.download()
    assert _rel(AqL, om.ax(got_p)) < AX_TOL
    # p.Ap block partials (one per block of elements; the buffer starts at zero)
    pL = om.scatter(got_p)
    pap = np.dot(pL, AqL)
    assert abs(parts.download().sum() - pap) <= 1e-12 * abs(pap)
    # first step (beta = 0) and no x update (alpha = 0)
    x2 = d["x"].download()
    gpu.cg_direction_ax(gm, own, 0.0, 0.0, d["r"], dinv, d["p"], pnew, d["x"], Aq, parts)
    assert _rel(pnew.download(), z) < 4e-16
    assert np.array_equal(d["x"].download(), x2)


@pytest.mark.parametrize("N,nrhs,precon", [(7, 4, True), (7, 2, False), (9, 4, True), (11, 4, True), (7, 1, True)])
def test_fused_step_fp32_packed_matches_unfused_operator(gpu, oracle, N, nrhs, precon):
    gm = gpu.Mesh(3, 2, 2, N=N, pert=0.1)
    Ng, E, Np = gm.Ngather, gm.E, gm.Np
    own = _owner(gpu, gm)
    v = gm.view
    ng = E * Np
    ops = {"wJ": gpu.DeviceBuffer(ng, np.float32), "ggeo": gpu.DeviceBuffer(6 * ng, np.float32),
           "gllw": gpu.DeviceBuffer(gm.Nq, np.float32), "D": gpu.DeviceBuffer(gm.Nq * gm.Nq, np.float32)}
    for name, n in (("wJ", ng), ("ggeo", 6 * ng), ("gllw", gm.Nq), ("D", gm.Nq * gm.Nq)):
        gpu.convert_f64_f32(getattr(v, name), n, ops[name])
    rng = np.random.default_rng(5)
    r = rng.uniform(-1, 1, Ng * nrhs).astype(np.float32)
    pold = rng.uniform(-1, 1, Ng * nrhs).astype(np.float32)
    x = rng.uniform(-1, 1, Ng * nrhs).astype(np.float32)
    invD = rng.uniform(0.5, 1.5, Ng).astype(np.float32) if precon else None
    alpha = [0.3, 0.0, -0.7, 1.1][:nrhs]
    beta = [0.9, 0.2, 0.0, 0.55][:nrhs]
    dr, dp, dx = (gpu.DeviceBuffer.from_host(a) for a in (r, pold, x))
    dinv = gpu.DeviceBuffer.from_host(invD) if precon else None
    pnew = gpu.DeviceBuffer(Ng * nrhs, np.float32)
    Aq = gpu.DeviceBuffer(gm.NL * nrhs, np.float32)
    parts = gpu.DeviceBuffer(nrhs * (E + 1))
    gpu.cg_direction_ax_f32_multi(gm, nrhs, own, ops, alpha, beta, dr, dinv, dp, pnew, dx, Aq, parts)
    z = (np.repeat(invD, nrhs) * r) if precon else r
    bl = np.tile(np.asarray(beta, np.float32), Ng)
    al = np.tile(np.asarray(alpha, np.float32), Ng)
    want_p = np.where(bl == 0, z, z + bl * pold)
    got_p = pnew.download()
    assert np.max(np.abs(got_p - want_p)) <= 4e-7 * np.max(np.abs(want_p))
    want_x = np.where(al == 0, x, al * pold + x)
    assert np.max(np.abs(dx.download() - want_x)) <= 4e-7 * np.max(np.abs(want_x))
    # the unfused operator in the same (TMA) form on the same p_new: the same bits
    Aq2 = gpu.DeviceBuffer(gm.NL * nrhs, np.float32)
    os.environ["BP_AX_VARIANT"] = "tma"
    try:
        gpu.ax_hex3d_f32_multi(gm, nrhs, pnew, Aq2, ops)
    finally:
        os.environ.pop("BP_AX_VARIANT", None)
    assert np.array_equal(Aq.download(), Aq2.download())


def _fp64_history(gpu, gm, fuse):
    # the TMA form in both runs (the autotuner might pick another form on a box this small)
    os.environ["BP_FUSE_DIRECTION"] = "1" if fuse else "0"
    os.environ["BP_AX_VARIANT"] = "tma"
    try:
        S = gpu.BP(gm, precon="JACOBI")
        b = S.rhs("RANDOM", 0)
        x = gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather))
        st, hr, ha = S.solve(x, b, tol=0.0, maxit=60)
        return st, hr, ha, x.download()
    finally:
        os.environ.pop("BP_FUSE_DIRECTION", None)
        os.environ.pop("BP_AX_VARIANT", None)


@pytest.mark.parametrize("N,Nf", [(7, 1), (5, 1), (3, 3)])
def test_fp64_cg_fused_matches_unfused_and_oracle(gpu, oracle, N, Nf):
    gm = gpu.Mesh(3, 3, 2, N=N, Nfields=Nf, pert=0.1)
    st1, hr1, ha1, x1 = _fp64_history(gpu, gm, True)
    st0, hr0, ha0, x0 = _fp64_history(gpu, gm, False)
    assert st1.iterations == st0.iterations == 60
    # per iteration while the residual is above 1e-6 r0 (deeper, CG amplifies
    # last-bit differences by about r0/r_k), then absolutely against r0
    live = hr0 >= 1e-6 * hr0[0]
    assert live[:20].all()
    assert np.max((np.abs(hr1 - hr0) / hr0)[live]) < 1e-12
    assert np.max((np.abs(ha1 - ha0) / np.abs(ha0))[live]) < 1e-12
    assert np.all(np.abs(hr1 - hr0) <= 1e-12 * hr0[0])
    assert _rel(x1, x0) < 1e-10
    assert st1.kernel_launches < st0.kernel_launches   # one kernel fewer per iteration
    om = oracle.Mesh(3, 3, 2, N, Nfields=Nf, pert=0.1)
    _, b_o = om.rhs_random(0)
    _, _, it, hr_o, _ = om.cg(b_o, 1.0, 0.0, 60, precon=True)
    live = hr_o >= 1e-6 * hr_o[0]
    assert np.max((np.abs(hr1 - hr_o) / hr_o)[live]) < HIST_TOL
    assert np.all(np.abs(hr1 - hr_o) <= HIST_TOL * hr_o[0])


def test_mixed_batch_fused_matches_unfused(gpu, oracle):
    res = {}
    for fuse in (True, False):
        os.environ["BP_FUSE_DIRECTION"] = "1" if fuse else "0"
        os.environ["BP_AX_VARIANT"] = "tma"
        try:
            B = gpu.Batch([{"nx": 4, "ny": 3, "nz": 3, "N": 7, "pert": 0.1, "pert_seed": 1, "nrhs": 4,
                            "rhs_seed": 0}], precon="JACOBI", precision="MIXED")
            stats, _ = B.solve(tol=1e-8, maxit=3000)
            res[fuse] = ([s.iterations for s in stats], [B.vectors(k)[0] for k in range(4)],
                         sum(s.kernel_launches for s in stats))
        finally:
            os.environ.pop("BP_FUSE_DIRECTION", None)
            os.environ.pop("BP_AX_VARIANT", None)
    om = oracle.Mesh(4, 3, 3, 7, pert=0.1)
    for k in range(4):
        _, b_o = om.rhs_random(k)
        for fuse in (True, False):
            xk = res[fuse][1][k]
            assert np.linalg.norm(b_o - om.operator(xk)) <= 1.0001e-8 * np.linalg.norm(b_o)
        # FP32 recursions in another rounding order: the same solution to the tolerance
        assert _rel(res[True][1][k], res[False][1][k]) < 1e-4
    assert all(abs(a - b) <= 3 for a, b in zip(res[True][0], res[False][0]))
    assert res[True][2] < res[False][2]   # one kernel fewer per iteration
