"""Parity at the benchmark sizes, CUDA path against the oracle.

The stored-factor BP5 box the headline is measured on (40^3 elements, p=7,
interior vertices perturbed by 0.1h with seed 1; 21,717,639 unknowns), the
same box under the over-integrated BP3 operator (9 Gauss points per
direction), and the BP6 box of 24^3 affine elements at p=15 with three fields
(138,804,837 unknowns).  The oracle runs on the host's cores (about a minute
in all).  Bars: numbering bit-exact; element operator and assembled operator
within 1e-12 relative (FP64); the gather of one E-vector bit-exact; the CG
residual history within 1e-10 per iteration while the residual is above
1e-6 r0.
"""
import hashlib

import numpy as np
import pytest

from test_gpu_parity import HIST_TOL, _check_history

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

AX_TOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i4").tobytes()).hexdigest()


@pytest.fixture(scope="module")
def box40(gpu, oracle):
    om = oracle.Mesh(40, 40, 40, 7, pert=0.1, pert_seed=1)
    gm = gpu.Mesh(40, 40, 40, N=7, pert=0.1, pert_seed=1)
    assert gm.Ngather == om.Ngather == 279 ** 3
    return om, gm


def test_box40_numbering_geometry_operator(gpu, oracle, box40):
    om, gm = box40
    for ours, theirs in (("GlobalToLocal", "G2L"), ("rowStarts", "rowStarts"), ("colIds", "colIds")):
        assert digest(gm.array(ours)) == digest(om.array(theirs)), ours
    # Factors computed on the device against the oracle's host values.  The
    # coordinate derivatives (about h/2 = 0.025) come from coordinates of size 1
    # through D entries up to 14: ~560 ulps of cancellation, so 1e-12 here.
    assert rel(gm.array("wJ"), om.array("wJ")) <= 1e-12
    assert rel(gm.array("ggeo"), om.array("ggeo")) <= 1e-12
    q = 2.0 * oracle.random(11, om.Ngather) - 1.0
    dq, dA = gpu.DeviceBuffer.from_host(q), gpu.DeviceBuffer(om.NL)
    gpu.ax_hex3d(gm, dq, dA)
    AqL_o = om.ax(q)
    assert rel(dA.download(), AqL_o) <= AX_TOL
    # the device gather of the oracle's own E-vector: bit for bit
    dv, dg = gpu.DeviceBuffer.from_host(AqL_o), gpu.DeviceBuffer(om.Ngather)
    gpu.ogs_gather(gm, dv, dg)
    Aq_o = om.gather(AqL_o)
    np.testing.assert_array_equal(dg.download(), Aq_o)
    S = gpu.BP(gm)
    dAq = gpu.DeviceBuffer(om.Ngather)
    S.operator(dq, dAq)
    assert rel(dAq.download(), Aq_o) <= AX_TOL


@pytest.mark.parametrize("precon", ["JACOBI", "NONE"])
def test_box40_cg_history(gpu, oracle, box40, precon):
    """100 iterations from x = 0 on b = M f, f = 2u-1 (seed 0): Jacobi-PCG (the
    benchmark's solver) and plain CG (the reference's cg::Solve)."""
    om, gm = box40
    _, b_o = om.rhs_random(0)
    x_o, _, it_o, hr_o, ha_o = om.cg(b_o, 1.0, 0.0, 100, precon=(precon == "JACOBI"))
    S = gpu.BP(gm, precon=precon)
    x = gpu.DeviceBuffer.from_host(np.zeros(om.Ngather))
    st, hr, ha = S.solve(x, S.rhs("RANDOM", 0), tol=0.0, maxit=100)
    assert st.iterations == it_o == 100
    live = _check_history(hr, hr_o)
    assert np.all((np.abs(ha - ha_o) / np.abs(ha_o))[live] < HIST_TOL)
    assert rel(x.download(), x_o) < 1e-9


def test_box40_bp3_operator(gpu, oracle, box40):
    """The over-integrated BP3 operator on the perturbed 40^3 box (Gauss-point
    factors computed on the device)."""
    om, gm = box40
    q = 2.0 * oracle.random(12, om.Ngather) - 1.0
    dq, dA = gpu.DeviceBuffer.from_host(q), gpu.DeviceBuffer(om.NL)
    gpu.ax_cub_hex3d(gm, 3, dq, dA)
    assert rel(dA.download(), om.ax(q, bp=3)) <= AX_TOL


def test_box24_p15_bp6_operator(gpu, oracle):
    """BP6: 24^3 affine elements, p=15, three fields."""
    om = oracle.Mesh(24, 24, 24, 15, affine=True, Nfields=3)
    gm = gpu.Mesh(24, 24, 24, N=15, affine=True, Nfields=3)
    assert gm.Ngather == om.Ngather == 3 * 359 ** 3
    assert digest(gm.array("GlobalToLocal")) == digest(om.array("G2L"))
    q = 2.0 * oracle.random(13, om.Ngather) - 1.0
    dq, dA = gpu.DeviceBuffer.from_host(q), gpu.DeviceBuffer(om.NL)
    gpu.ax_hex3d(gm, dq, dA)
    AqL_o = om.ax(q, bp=6)
    assert rel(dA.download(), AqL_o) <= AX_TOL
    del dA
    S = gpu.BP(gm, bp=6)
    dAq = gpu.DeviceBuffer(om.Ngather)
    S.operator(dq, dAq)
    assert rel(dAq.download(), om.gather(AqL_o)) <= AX_TOL
