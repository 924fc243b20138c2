"""The tensor-core affine operator (bp_ax_mma.cu) at degree 15, against the oracle.

At Nq = 16 the affine BP5/BP6 operator runs its contractions as warp MMAs:
DMMA (m8n8k4 f64) in FP64 and split-operand TF32 (m16n8k8, two TF32 parts per
operand, FP32 accumulation) in FP32.  Bars: FP64 within 1e-12 of the oracle's
FP64 operator (the parity bar); FP32 within 2e-6 (FP32 rounding of the inputs,
the factors and the sums; plain TF32 would be about 3e-4); fused p.Ap inside
CG (the residual history within 1e-10 of the oracle per iteration); a mixed
solve to 1e-8 checked with the FP64 operator.
"""
import numpy as np
import pytest

from test_gpu_parity import HIST_TOL, _check_history

pytestmark = pytest.mark.gpu

CASES = [(2, 2, 2, 1), (3, 2, 2, 1), (2, 2, 1, 3), (3, 2, 2, 3)]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("nx,ny,nz,Nf", CASES)
def test_mma_fp64_operator_matches_oracle(gpu, oracle, nx, ny, nz, Nf):
    om = oracle.Mesh(nx, ny, nz, 15, affine=True, Nfields=Nf)
    gm = gpu.Mesh(nx, ny, nz, N=15, affine=True, Nfields=Nf)
    for seed in (1, 2):
        q = 2.0 * oracle.random(seed, om.Ngather) - 1.0
        dq, dA = gpu.DeviceBuffer.from_host(q), gpu.DeviceBuffer(om.NL)
        gpu.ax_hex3d(gm, dq, dA)
        assert rel(dA.download(), om.ax(q, bp=6 if Nf == 3 else 5)) <= 1e-12


@pytest.mark.parametrize("nx,ny,nz,Nf", CASES)
def test_mma_fp32_operator_matches_oracle(gpu, oracle, nx, ny, nz, Nf):
    om = oracle.Mesh(nx, ny, nz, 15, affine=True, Nfields=Nf)
    gm = gpu.Mesh(nx, ny, nz, N=15, affine=True, Nfields=Nf)
    v = gm.view
    ops = {k: gpu.DeviceBuffer(n, np.float32) for k, n in
           (("wJ", gm.E), ("ggeo", 6 * gm.E), ("gllw", gm.Nq), ("D", gm.Nq * gm.Nq))}
    for name, n in (("wJ", gm.E), ("ggeo", 6 * gm.E), ("gllw", gm.Nq), ("D", gm.Nq * gm.Nq)):
        gpu.convert_f64_f32(getattr(v, name), n, ops[name])
    q = 2.0 * oracle.random(4, om.Ngather) - 1.0
    q32 = gpu.DeviceBuffer.from_host(q.astype(np.float32))
    A32 = gpu.DeviceBuffer(om.NL, np.float32)
    gpu.ax_hex3d_f32(gm, q32, A32, ops)
    want = om.ax(q.astype(np.float32).astype(np.float64), bp=6 if Nf == 3 else 5)
    err = rel(A32.download().astype(np.float64), want)
    assert err <= 2e-6, err


@pytest.mark.parametrize("precon", ["JACOBI", "NONE"])
def test_mma_operator_inside_cg(gpu, oracle, precon):
    om = oracle.Mesh(3, 3, 2, 15, affine=True)
    gm = gpu.Mesh(3, 3, 2, N=15, affine=True)
    _, b_o = om.rhs_random(0)
    x_o, _, it_o, hr_o, ha_o = om.cg(b_o, 1.0, 0.0, 60, precon=(precon == "JACOBI"))
    S = gpu.BP(gm, precon=precon)
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    st, hr, ha = S.solve(x, S.rhs("RANDOM", 0), tol=0.0, maxit=60)
    assert st.iterations == it_o == 60
    live = _check_history(hr, hr_o)
    assert np.all((np.abs(ha - ha_o) / np.abs(ha_o))[live] < HIST_TOL)


def test_mma_mixed_solve_reaches_tolerance(gpu, oracle):
    om = oracle.Mesh(3, 3, 3, 15, affine=True, Nfields=3)
    gm = gpu.Mesh(3, 3, 3, N=15, affine=True, Nfields=3)
    S = gpu.BP(gm, precon="JACOBI", precision="MIXED")
    S64 = gpu.BP(gm, precon="JACOBI")
    _, b_o = om.rhs_random(0)
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    st, _, _ = S.solve(x, gpu.DeviceBuffer.from_host(b_o), tol=1e-8, maxit=20000)
    Ax = gpu.DeviceBuffer(om.Ngather)
    S64.operator(x, Ax)
    assert np.linalg.norm(b_o - Ax.download()) / np.linalg.norm(b_o) <= 1.0001e-8
    _, _, it_o, _, _ = om.cg(b_o, 1.0, 1e-8, 20000, precon=True)
    assert st.iterations <= 1.25 * it_o + 20, (st.iterations, it_o)


def test_mma_packed_p7_operator_when_selected(gpu, oracle, monkeypatch):
    """The packed four-rhs FP32 form at p=7 (BP_AX_VARIANT=mma; the TMA form is
    the default there, being faster): each lane equals the FP64 oracle's
    operator to FP32 accuracy and the default form to 1e-6."""
    om = oracle.Mesh(3, 2, 2, 7, pert=0.1)
    gm = gpu.Mesh(3, 2, 2, N=7, pert=0.1)
    v = gm.view
    ng = gm.E * gm.Np
    ops = {"wJ": gpu.DeviceBuffer(ng, np.float32), "ggeo": gpu.DeviceBuffer(6 * ng, np.float32),
           "gllw": gpu.DeviceBuffer(gm.Nq, np.float32), "D": gpu.DeviceBuffer(gm.Nq * gm.Nq, np.float32)}
    for name, n in (("wJ", ng), ("ggeo", 6 * ng), ("gllw", gm.Nq), ("D", gm.Nq * gm.Nq)):
        gpu.convert_f64_f32(getattr(v, name), n, ops[name])
    Q = np.stack([2 * oracle.random(30 + k, gm.Ngather) - 1 for k in range(4)], axis=1).astype(np.float32)
    dq = gpu.DeviceBuffer.from_host(np.ascontiguousarray(Q).ravel())
    out = {}
    for form in ("mma", "tma"):
        monkeypatch.setenv("BP_AX_VARIANT", form)
        dA = gpu.DeviceBuffer(gm.NL * 4, np.float32)
        gpu.ax_hex3d_f32_multi(gm, 4, dq, dA, ops)
        out[form] = dA.download().reshape(gm.NL, 4)
    monkeypatch.delenv("BP_AX_VARIANT")
    for k in range(4):
        want = om.ax(Q[:, k].astype(np.float64))
        assert rel(out["mma"][:, k].astype(np.float64), want) <= 2e-6
        assert rel(out["mma"][:, k], out["tma"][:, k]) <= 1e-6
