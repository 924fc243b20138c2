"""Tri2D parity pinned to the reference's OWN code, on the CPU.

The fixtures tests/golden/ref_tri_*.npz were written by the reference's host
set-up compiled here (libs/mesh meshBasisTri2D.cpp, meshReferenceNodesTri2D.cpp,
meshSetupBoxTri2D.cpp, meshGeometricFactorsTri2D.cpp, meshConnectNodes.cpp,
meshMaskedGatherScatterSetup.cpp, libs/ogs; generator
tests/golden/make_golden.py).  Held to them: the oracle's numpy restatement
(oracle/tri2d.py) and the library's own host code (bp_basis_tri2d,
bp_box_numbering with simplex = 1).  Integers, gather and scatter bit-exact;
node coordinates, D, MM, S, geometric factors within FP_TOL(N) of the largest
entry (the reference inverts its Vandermonde matrices through LAPACK stand-ins,
the oracle through numpy, the library through its own Gauss-Jordan).
"""
import glob
import os

import numpy as np
import pytest

from test_ref_golden import FP_TOL, digest, rel

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TRI = sorted(glob.glob(os.path.join(GOLDEN, "ref_tri_*.npz")))
FULL = [f for f in TRI if "sha256_GlobalToLocal" in np.load(f).files]
SMALL = [f for f in TRI if f not in FULL]


def case(path):
    """(fixture, nx, ny, N)."""
    g = np.load(path)
    cli = str(g["cli"]).split()
    opts = {cli[i]: int(cli[i + 1]) for i in range(len(cli) - 1) if cli[i] in ("-nx", "-ny", "-p")}
    assert "Tri" in cli and "-a" in cli
    return g, opts["-nx"], opts["-ny"], opts["-p"]


def ids(paths):
    return [os.path.basename(p)[8:-4] for p in paths]


@pytest.fixture(scope="module")
def tri():
    from oracle import tri2d
    return tri2d


@pytest.mark.parametrize("path", SMALL, ids=ids(SMALL))
def test_oracle_matches_reference_code(tri, path):
    g, nx, ny, N = case(path)
    m = tri.Mesh(nx, ny, N)
    Np = m.Np
    assert (m.E, m.Np, m.Ngather) == (int(g["Nelements"][0]), int(g["Np"][0]), int(g["Ngather"][0]))
    np.testing.assert_array_equal(m.EToV, g["EToV"])
    assert rel(m.EX, g["EX"]) <= 1e-15 and rel(m.EY, g["EY"]) <= 1e-15
    assert rel(m.x.ravel(), g["x"]) <= FP_TOL(N) and rel(m.y.ravel(), g["y"]) <= FP_TOL(N)
    D = g["D"].reshape(2, Np, Np)
    assert rel(m.Dr, D[0]) <= FP_TOL(N) and rel(m.Ds, D[1]) <= FP_TOL(N)
    assert rel(m.MM, g["MM"].reshape(Np, Np)) <= FP_TOL(N)
    S = g["S"].reshape(3, Np, Np)
    for k, mine in enumerate((m.Srr, m.Srs, m.Sss)):
        assert rel(mine, S[k]) <= FP_TOL(N), k
    assert rel(m.wJ, g["wJ"]) <= 1e-14 and rel(m.ggeo.ravel(), g["ggeo"]) <= 1e-14
    np.testing.assert_array_equal(m.globalIds, g["globalIds"])
    np.testing.assert_array_equal(m.G2L, g["GlobalToLocal"])
    np.testing.assert_array_equal(m.rowStarts, g["rowStartsT"])
    np.testing.assert_array_equal(m.colIds, g["colIdsT"])
    np.testing.assert_array_equal(m.gather(g["gather_in"]), g["gather_out"])
    np.testing.assert_array_equal(m.scatter(g["scatter_in"]), g["scatter_out"])


@pytest.mark.parametrize("path", SMALL, ids=ids(SMALL))
def test_library_host_setup_matches_reference_code(bp, path):
    g, nx, ny, N = case(path)
    r, s, Dr, Ds, MM, Srr, Srs, Sss = bp.basis_tri2d(N)
    Np = r.size
    D = g["D"].reshape(2, Np, Np)
    assert rel(Dr, D[0]) <= FP_TOL(N) and rel(Ds, D[1]) <= FP_TOL(N)
    assert rel(MM, g["MM"].reshape(Np, Np)) <= FP_TOL(N)
    S = g["S"].reshape(3, Np, Np)
    for k, mine in enumerate((Srr, Srs, Sss)):
        assert rel(mine, S[k]) <= FP_TOL(N), k
    g2l, rs, ci = bp.box_numbering(nx, ny, 1, N, dim=2, simplex=True)
    np.testing.assert_array_equal(g2l, g["GlobalToLocal"])
    np.testing.assert_array_equal(rs, g["rowStartsT"])
    np.testing.assert_array_equal(ci, g["colIdsT"])


@pytest.mark.parametrize("path", FULL, ids=ids(FULL))
def test_library_numbering_full_size_matches_reference_code(bp, path):
    g, nx, ny, N = case(path)
    g2l, rs, ci = bp.box_numbering(nx, ny, 1, N, dim=2, simplex=True)
    for a, k in ((g2l, "GlobalToLocal"), (rs, "rowStartsT"), (ci, "colIdsT")):
        assert a.size == int(g["size_" + k]), k
        assert digest(a.astype("<i4")) == str(g["sha256_" + k]), k


@pytest.mark.parametrize("N", [1, 2, 5, 9, 15])
def test_reference_element_known_answers(tri, N):
    # the mass matrix integrates 1 to the reference triangle's area (2), S
    # annihilates constants, Dr and Ds differentiate r and s exactly
    r, s, Dr, Ds, MM, Srr, Srs, Sss = tri.reference_matrices(N)
    one = np.ones_like(r)
    assert abs(one @ MM @ one - 2.0) < 1e-12
    for S in (Srr, Srs, Sss):
        assert np.max(np.abs(S @ one)) < 1e-9 * np.max(np.abs(S))
        assert np.max(np.abs(S - S.T)) < 1e-9 * np.max(np.abs(S))
    assert np.max(np.abs(Dr @ r - 1)) < 1e-9 and np.max(np.abs(Ds @ s - 1)) < 1e-9
    assert np.max(np.abs(Dr @ s)) < 1e-9 and np.max(np.abs(Ds @ r)) < 1e-9
