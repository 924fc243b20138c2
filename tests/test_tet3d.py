"""Tet3D parity pinned to the reference's OWN code, on the CPU.

The fixtures tests/golden/ref_tet_*.npz were written by the reference's host
set-up compiled here (libs/mesh meshBasisTet3D.cpp, meshReferenceNodesTet3D.cpp,
meshSetupBoxTet3D.cpp, meshGeometricFactorsTet3D.cpp, meshConnectNodes.cpp,
meshMaskedGatherScatterSetup.cpp, libs/ogs; generator
tests/golden/make_golden.py).  Held to them: the oracle's numpy restatement
(oracle/tet3d.py) and the library's own host code (bp_basis_tet3d,
bp_box_numbering with dim 3 and simplex 1).  Integers, gather and scatter
bit-exact; node coordinates, D, MM, S and geometric factors within FP_TOL(N),
widened to 5e-16 Np for the matrices: their inverses of Np x Np Vandermonde
products (Np = 120 at p = 7) differ in the last bits between the reference's
LAPACK stand-ins, numpy and the library's Gauss-Jordan.
"""
import glob
import os

import numpy as np
import pytest

from test_ref_golden import FP_TOL, digest, rel

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TET = sorted(glob.glob(os.path.join(GOLDEN, "ref_tet_*.npz")))
FULL = [f for f in TET if "sha256_GlobalToLocal" in np.load(f).files]
SMALL = [f for f in TET if f not in FULL]


def mtol(N, Np):
    return max(FP_TOL(N), 5e-16 * Np)


def case(path):
    """(fixture, nx, ny, nz, N)."""
    g = np.load(path)
    cli = str(g["cli"]).split()
    opts = {cli[i]: int(cli[i + 1]) for i in range(len(cli) - 1) if cli[i] in ("-nx", "-ny", "-nz", "-p")}
    assert "Tet" in cli and "-a" in cli
    return g, opts["-nx"], opts["-ny"], opts["-nz"], opts["-p"]


def ids(paths):
    return [os.path.basename(p)[8:-4] for p in paths]


@pytest.fixture(scope="module")
def tet():
    from oracle import tet3d
    return tet3d


@pytest.mark.parametrize("path", SMALL, ids=ids(SMALL))
def test_oracle_matches_reference_code(tet, path):
    g, nx, ny, nz, N = case(path)
    m = tet.Mesh(nx, ny, nz, N)
    Np = m.Np
    assert (m.E, m.Np, m.Ngather) == (int(g["Nelements"][0]), int(g["Np"][0]), int(g["Ngather"][0]))
    np.testing.assert_array_equal(m.EToV, g["EToV"])
    for mine, k in ((m.EX, "EX"), (m.EY, "EY"), (m.EZ, "EZ")):
        assert rel(mine, g[k]) <= 1e-15, k
    for mine, k in ((m.x, "x"), (m.y, "y"), (m.z, "z")):
        assert rel(mine.ravel(), g[k]) <= FP_TOL(N), k
    D = g["D"].reshape(3, Np, Np)
    for a, mine in enumerate((m.Dr, m.Ds, m.Dt)):
        assert rel(mine, D[a]) <= mtol(N, Np), a
    assert rel(m.MM, g["MM"].reshape(Np, Np)) <= mtol(N, Np)
    assert rel(m.S, g["S"].reshape(6, Np, Np)) <= mtol(N, Np)
    assert rel(m.wJ, g["wJ"]) <= 1e-14 and rel(m.ggeo.ravel(), g["ggeo"]) <= 1e-14
    np.testing.assert_array_equal(m.globalIds, g["globalIds"])
    np.testing.assert_array_equal(m.G2L, g["GlobalToLocal"])
    np.testing.assert_array_equal(m.rowStarts, g["rowStartsT"])
    np.testing.assert_array_equal(m.colIds, g["colIdsT"])
    np.testing.assert_array_equal(m.gather(g["gather_in"]), g["gather_out"])
    np.testing.assert_array_equal(m.scatter(g["scatter_in"]), g["scatter_out"])


@pytest.mark.parametrize("path", SMALL, ids=ids(SMALL))
def test_library_host_setup_matches_reference_code(bp, path):
    g, nx, ny, nz, N = case(path)
    r, s, t, Dr, Ds, Dt, MM, S = bp.basis_tet3d(N)
    Np = r.size
    D = g["D"].reshape(3, Np, Np)
    for a, mine in enumerate((Dr, Ds, Dt)):
        assert rel(mine, D[a]) <= mtol(N, Np), a
    assert rel(MM, g["MM"].reshape(Np, Np)) <= mtol(N, Np)
    assert rel(S, g["S"].reshape(6, Np, Np)) <= mtol(N, Np)
    g2l, rs, ci = bp.box_numbering(nx, ny, nz, N, dim=3, simplex=True)
    np.testing.assert_array_equal(g2l, g["GlobalToLocal"])
    np.testing.assert_array_equal(rs, g["rowStartsT"])
    np.testing.assert_array_equal(ci, g["colIdsT"])


@pytest.mark.parametrize("path", FULL, ids=ids(FULL))
def test_library_numbering_full_size_matches_reference_code(bp, path):
    g, nx, ny, nz, N = case(path)
    g2l, rs, ci = bp.box_numbering(nx, ny, nz, N, dim=3, simplex=True)
    for a, k in ((g2l, "GlobalToLocal"), (rs, "rowStartsT"), (ci, "colIdsT")):
        assert a.size == int(g["size_" + k]), k
        assert digest(a.astype("<i4")) == str(g["sha256_" + k]), k


@pytest.mark.parametrize("N", [1, 2, 5, 8])
def test_reference_element_known_answers(tet, N):
    # MM integrates 1 to the reference tetrahedron's volume (4/3); the S_ab
    # annihilate constants and are symmetric; D differentiates r, s, t exactly
    r, s, t, Dr, Ds, Dt, MM, S = tet.reference_matrices(N)
    one = np.ones_like(r)
    assert abs(one @ MM @ one - 4.0 / 3.0) < 1e-12
    for X in S:
        assert np.max(np.abs(X @ one)) < 1e-9 * np.max(np.abs(X))
        assert np.max(np.abs(X - X.T)) < 1e-9 * np.max(np.abs(X))
    for Da, c in ((Dr, r), (Ds, s), (Dt, t)):
        assert np.max(np.abs(Da @ c - 1)) < 1e-9
