"""Host side of the over-integrated operators (no GPU): the library's 1D
cubature data against the oracle, and the oracle's BP1-BP4 operators against
properties they must have."""
import numpy as np
import pytest


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("N", [1, 2, 3, 5, 7, 10, 15])
def test_basis_cubature_matches_oracle(bp, oracle, N):
    c = bp.basis_cubature(N)
    ma = oracle.Mesh(1, 1, 1, N, affine=True)
    mc = oracle.Mesh(1, 1, 1, N)
    assert _rel(c["r"], ma.array("cubr")) < 1e-15
    assert _rel(c["w"], ma.array("cubw")) < 1e-14
    assert _rel(c["I"].ravel(), ma.array("cubInterp")) < 1e-13
    assert _rel(c["D"].ravel(), mc.array("cubD")) < 1e-13
    assert _rel(c["invV"].ravel(), ma.array("invV")) < 1e-13
    assert _rel(c["Dmodal"].ravel(), ma.array("cubD")) < 1e-13
    assert _rel(c["MM"].ravel(), ma.array("MM")) < 1e-13
    # Gauss rule with N+2 points integrates degree 2N+3 exactly
    for d in range(0, 2 * N + 4):
        exact = 0.0 if d % 2 else 2.0 / (d + 1)
        assert abs(np.sum(c["w"] * c["r"] ** d) - exact) < 1e-13


def test_basis_cubature_bad_degree(bp):
    with pytest.raises(bp.BPError):
        bp.basis_cubature(0)
    with pytest.raises(bp.BPError):
        bp.basis_cubature(16)


@pytest.mark.parametrize("N,Nf", [(1, 1), (2, 3), (3, 1), (5, 1), (5, 3)])
def test_oracle_affine_and_curved_agree_on_a_box(oracle, N, Nf):
    # on the undeformed box the modal affine operators (exact integration) and
    # the curved Gauss-point operators (exact for these integrands) coincide
    ma = oracle.Mesh(2, 2, 3, N, affine=True, Nfields=Nf)
    mc = oracle.Mesh(2, 2, 3, N, affine=False, Nfields=Nf)
    q = 2 * oracle.random(7, ma.Ngather) - 1
    for bp in ((1, 3) if Nf == 1 else (2, 4)):
        assert _rel(ma.operator(q, 1.0, bp), mc.operator(q, 1.0, bp)) < 1e-13
        assert _rel(ma.jacobi_diag(1.0, bp), mc.jacobi_diag(1.0, bp)) < 1e-13


@pytest.mark.parametrize("bp,affine", [(1, False), (1, True), (3, False), (3, True)])
def test_oracle_cub_operator_symmetric_and_diagonal(oracle, bp, affine):
    m = oracle.Mesh(2, 2, 2, 3, affine=affine, pert=0.0 if affine else 0.15)
    rng = np.random.default_rng(0)
    u, v = rng.standard_normal(m.Ngather), rng.standard_normal(m.Ngather)
    uAv, vAu = u @ m.operator(v, 1.0, bp), v @ m.operator(u, 1.0, bp)
    assert abs(uAv - vAu) <= 1e-13 * abs(uAv)
    assert u @ m.operator(u, 1.0, bp) > 0
    d = m.jacobi_diag(1.0, bp)
    E = np.eye(m.Ngather)
    probe = np.array([m.operator(E[i], 1.0, bp)[i] for i in range(0, m.Ngather, 3)])
    assert _rel(probe, d[::3]) < 1e-13
