"""Host-side logic of the product library against the oracle, on the CPU.

The numbering (GlobalToLocal, CSR rowStarts/colIds) must be bit-exact with
the reference's algorithm (libs/ogs/ogsSetup.cpp:492-579, 833-849 and
libs/mesh/meshConnectNodes.cpp:32-82), which the oracle restates with generic
connectivity while the library derives it in closed form from the box.
"""
import numpy as np
import pytest


CASES = [(1, 1, 1, 1, 1), (2, 2, 2, 1, 1), (1, 1, 1, 4, 1), (3, 2, 4, 2, 1), (2, 3, 2, 3, 3), (4, 4, 4, 4, 1),
         (2, 2, 3, 7, 1), (1, 2, 1, 5, 3), (5, 1, 2, 3, 1), (2, 2, 2, 9, 1), (1, 1, 2, 15, 1), (3, 3, 3, 2, 3)]


@pytest.mark.parametrize("nx,ny,nz,N,Nf", CASES)
def test_numbering_bit_exact(bp, oracle, nx, ny, nz, N, Nf):
    g2l, rs, ci = bp.box_numbering(nx, ny, nz, N, Nf)
    m = oracle.Mesh(nx, ny, nz, N, Nfields=Nf)
    np.testing.assert_array_equal(g2l, m.array("G2L"))
    np.testing.assert_array_equal(rs, m.array("rowStarts"))
    np.testing.assert_array_equal(ci, m.array("colIds"))


@pytest.mark.parametrize("N", list(range(1, 16)))
def test_basis_matches_oracle(bp, oracle, N):
    z, w, D = bp.basis_gll(N)
    zo, wo = oracle.jacobi_gll(N)
    Do = oracle.dmatrix1d(N, zo, zo)
    np.testing.assert_allclose(z, zo, atol=2e-15)
    np.testing.assert_allclose(w, wo, rtol=2e-13)
    np.testing.assert_allclose(D, Do, atol=1e-12 * max(1.0, np.abs(Do).max()))


@pytest.mark.parametrize("pert,seed", [(0.0, 1), (0.1, 1), (0.25, 9)])
def test_vertices_match_oracle(bp, oracle, pert, seed):
    ex, ey, ez = bp.box_vertices(4, 3, 5, pert=pert, pert_seed=seed)
    m = oracle.Mesh(4, 3, 5, 1, pert=pert, pert_seed=seed)
    np.testing.assert_array_equal(ex, m.array("EX"))
    np.testing.assert_array_equal(ey, m.array("EY"))
    np.testing.assert_array_equal(ez, m.array("EZ"))


def test_numbering_rejects_bad_sizes(bp):
    with pytest.raises(bp.BPError):
        bp.box_numbering(0, 1, 1, 2)
    with pytest.raises(bp.BPError):
        bp.box_numbering(1, 1, 1, 16)
    with pytest.raises(bp.BPError):
        bp.box_numbering(1, 1, 1, 2, Nfields=2)
    # E*Np*Nfields beyond int32 (dlong) is refused, not wrapped
    with pytest.raises(bp.BPError):
        bp.box_numbering(100, 100, 100, 15)


def test_uneven_problem_set(bp, oracle):
    # the LCG matches the reference's (the oracle's restatement)
    np.testing.assert_array_equal(np.array(bp.lcg_uniform(7, 50)), oracle.random(7, 50))
    P = bp.uneven_problems()
    assert len(P) == 64 and all(p["nrhs"] == 4 for p in P)
    assert {p["N"] for p in P} == set(range(3, 11))
    assert min(p["nx"] for p in P) >= 8 and max(p["nx"] for p in P) <= 24
    assert [p["pert_seed"] for p in P] == list(range(100, 164))
    assert [p["rhs_seed"] for p in P] == [1000 + 4 * i for i in range(64)]
