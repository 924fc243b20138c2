"""Parity pinned to the reference's OWN code, on the CPU.

The fixtures in tests/golden/ were written by the reference's host sources
(libs/mesh, libs/ogs, libs/primitives, libs/core, compiled where they lie with
the one-rank MPI / host OCCA / LAPACK shims of oracle/ref_shim/; generator:
tests/golden/make_golden.py).  They hold the reference's masked numbering
(mesh_t::MaskedGatherScatterSetup + ogs_t::Setup + SetupGlobalToLocalMapping),
its gather CSR, basis, geometric factors and cubature data, and its host ogs
Gather (Add, Trans) and Scatter (NoTrans) applied to seeded vectors.

Bars: every integer array bit-exact; gather and scatter bit-exact; FP64 basis,
geometry and cubature data within FP_TOL(N) relative to the array's largest
entry.  FP_TOL is 2e-14 up to degree 7 and 3e-13 at higher degree: the
reference builds its GLL/Gauss nodes with a LAPACK eigen-solve and its
differentiation and interpolation matrices with Vandermonde solves (stand-ins
here, the system LAPACK being absent), the oracle and the library with Newton
iterations and closed forms; the last-bit differences of the nodes grow with
the conditioning of the degree-15 Vandermonde systems.
"""
import glob
import hashlib
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# Hex3D and Quad2D fixtures (the simplex ones, ref_tri_* and ref_tet_*, are read by
# tests/test_tri2d.py and tests/test_tet3d.py)
FILES = sorted(f for f in glob.glob(os.path.join(GOLDEN, "ref_*.npz"))
               if not os.path.basename(f).startswith(("ref_tri_", "ref_tet_")))
FULL = [f for f in FILES if "sha256_GlobalToLocal" in np.load(f).files]
SMALL = [f for f in FILES if f not in FULL]


def FP_TOL(N):
    return 2e-14 if N <= 7 else 3e-13


def case(path):
    """(fixture, nx, ny, nz, N, affine, Nfields, dim); Quad2D cases (-e Quad) have dim 2 and nz 1."""
    g = np.load(path)
    cli = str(g["cli"]).split()
    opts = {cli[i]: int(cli[i + 1]) for i in range(len(cli) - 1) if cli[i] in ("-nx", "-ny", "-nz", "-p")}
    dim = 2 if "Quad" in cli else 3
    nz = opts["-nz"] if dim == 3 else 1
    return g, opts["-nx"], opts["-ny"], nz, opts["-p"], "-a" in cli, int(g["Nfields"][0]), dim


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    assert a.shape == b.shape, (a.shape, b.shape)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def ids(paths):
    return [os.path.basename(p)[4:-4] for p in paths]


def test_fixtures_present():
    assert len(SMALL) >= 6 and len(FULL) >= 1
    assert sum("quad" in f for f in SMALL) >= 4 and sum("quad" in f for f in FULL) >= 1


@pytest.mark.parametrize("path", SMALL, ids=ids(SMALL))
def test_oracle_matches_reference_code(oracle, path):
    g, nx, ny, nz, N, affine, nf, dim = case(path)
    m = oracle.Mesh(nx, ny, nz, N, affine=affine, Nfields=nf, dim=dim)
    assert (m.E, m.Np, m.Ngather) == (int(g["Nelements"][0]), int(g["Np"][0]), int(g["Ngather"][0]))
    for ours, theirs in (("G2L", "GlobalToLocal"), ("rowStarts", "rowStartsT"), ("colIds", "colIdsT"),
                         ("globalIds", "globalIds"), ("EToV", "EToV"), ("EX", "EX"), ("EY", "EY"), ("EZ", "EZ")):
        np.testing.assert_array_equal(m.array(ours), g[theirs], err_msg=theirs)
    if dim == 2:   # the Quad2D restatement covers the BP5/BP6 data (no over-integration)
        names = ["gllz", "gllw", "D", "MM", "x", "y", "wJ", "ggeo"]
    else:
        names = ["gllz", "gllw", "D", "MM", "x", "y", "z", "wJ", "ggeo", "cubr", "cubw", "cubInterp", "cubD"]
        names += ["invV"] if affine else ["cubwJ", "cubggeo"]
    for k in names:
        assert rel(m.array(k), g[k]) <= FP_TOL(N), k
    np.testing.assert_array_equal(m.gather(g["gather_in"]), g["gather_out"])
    np.testing.assert_array_equal(m.scatter(g["scatter_in"]), g["scatter_out"])


@pytest.mark.parametrize("path", SMALL, ids=ids(SMALL))
def test_library_host_setup_matches_reference_code(bp, path):
    g, nx, ny, nz, N, affine, nf, dim = case(path)
    g2l, rs, ci = bp.box_numbering(nx, ny, nz, N, nf, dim=dim)
    np.testing.assert_array_equal(g2l, g["GlobalToLocal"])
    np.testing.assert_array_equal(rs, g["rowStartsT"])
    np.testing.assert_array_equal(ci, g["colIdsT"])
    ex, ey, ez = bp.box_vertices(nx, ny, nz, dim=dim)
    for a, k in ((ex, "EX"), (ey, "EY"), (ez, "EZ")):
        np.testing.assert_array_equal(a, g[k], err_msg=k)
    z, w, D = bp.basis_gll(N)
    assert rel(z, g["gllz"]) <= FP_TOL(N) and rel(w, g["gllw"]) <= FP_TOL(N)
    assert rel(D.ravel(), g["D"]) <= FP_TOL(N)
    if dim == 2:
        return
    c = bp.basis_cubature(N)
    assert rel(c["r"], g["cubr"]) <= FP_TOL(N) and rel(c["w"], g["cubw"]) <= FP_TOL(N)
    assert rel(c["I"].ravel(), g["cubInterp"]) <= FP_TOL(N)
    assert rel(c["MM"].ravel(), g["MM"]) <= FP_TOL(N)
    if affine:
        assert rel(c["invV"].ravel(), g["invV"]) <= FP_TOL(N)
        assert rel(c["Dmodal"].ravel(), g["cubD"]) <= FP_TOL(N)
    else:
        assert rel(c["D"].ravel(), g["cubD"]) <= FP_TOL(N)


@pytest.mark.parametrize("path", FULL, ids=ids(FULL))
def test_full_size_numbering_matches_reference_code(bp, oracle, path):
    """The BP5 p=4 box of 16^3 affine elements (250,047 unknowns) and a Quad2D box of 64 x 48 p=6 elements:
    the numbering and CSR of the library's host form and of the oracle hash to the reference's own arrays."""
    g, nx, ny, nz, N, affine, nf, dim = case(path)
    g2l, rs, ci = bp.box_numbering(nx, ny, nz, N, nf, dim=dim)
    m = oracle.Mesh(nx, ny, nz, N, affine=affine, Nfields=nf, dim=dim)
    for arrays in ((g2l, rs, ci), (m.array("G2L"), m.array("rowStarts"), m.array("colIds"))):
        for a, k in zip(arrays, ("GlobalToLocal", "rowStartsT", "colIdsT")):
            assert a.size == int(g["size_" + k]), k
            assert digest(a.astype("<i4")) == str(g["sha256_" + k]), k
    z, w, D = bp.basis_gll(N)
    assert rel(D.ravel(), g["D"]) <= FP_TOL(N)
