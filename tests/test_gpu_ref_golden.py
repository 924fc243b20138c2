"""Parity pinned to the reference's OWN code, on the GPU.

The device-built mesh (bp_mesh_create: box, numbering on the device,
geometric factors on the device; bp_mesh_cubature) and the device gather and
scatter kernels against the fixtures the reference's host sources wrote
(tests/golden/, generator tests/golden/make_golden.py).  Bars as in
test_ref_golden.py: integers, gather and scatter bit-exact; FP64 data within
FP_TOL(N) of the largest entry.
"""
import numpy as np
import pytest

from test_ref_golden import FP_TOL, FULL, SMALL, case, digest, ids, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", SMALL, ids=ids(SMALL))
def test_device_mesh_matches_reference_code(gpu, path):
    g, nx, ny, nz, N, affine, nf, dim = case(path)
    m = gpu.Mesh(nx, ny, nz, N=N, affine=affine, Nfields=nf, dim=dim)
    assert (m.E, m.Np, m.Ngather) == (int(g["Nelements"][0]), int(g["Np"][0]), int(g["Ngather"][0]))
    np.testing.assert_array_equal(m.array("GlobalToLocal"), g["GlobalToLocal"])
    np.testing.assert_array_equal(m.array("rowStarts"), g["rowStartsT"])
    np.testing.assert_array_equal(m.array("colIds"), g["colIdsT"])
    for k in ("EX", "EY", "EZ")[:dim]:
        np.testing.assert_array_equal(m.array(k), g[k], err_msg=k)
    # Quad2D meshes carry no cubature data (BP5/BP6 only)
    cub = ("cubr", "cubw", "cubInterp", "cubD", "MM") if dim == 3 else ()
    for k in ("gllz", "gllw", "D", "wJ", "ggeo") + cub:
        assert rel(m.array(k), g[k]) <= FP_TOL(N), k
    if dim == 3:
        for k in (("invV",) if affine else ("cubwJ", "cubggeo")):
            assert rel(m.array(k), g[k]) <= FP_TOL(N), k

    # the device gather (Add, Trans) and scatter (NoTrans) against the reference's host ones
    v = gpu.DeviceBuffer.from_host(g["gather_in"])
    gv = gpu.DeviceBuffer(m.Ngather)
    gpu.ogs_gather(m, v, gv)
    np.testing.assert_array_equal(gv.download(), g["gather_out"])
    s = gpu.DeviceBuffer.from_host(g["scatter_in"])
    sv = gpu.DeviceBuffer(m.NL)
    sv.zero()
    gpu.ogs_scatter(m, s, sv)
    np.testing.assert_array_equal(sv.download(), g["scatter_out"])


@pytest.mark.parametrize("path", FULL, ids=ids(FULL))
def test_device_numbering_full_size_matches_reference_code(gpu, path):
    g, nx, ny, nz, N, affine, nf, dim = case(path)
    m = gpu.Mesh(nx, ny, nz, N=N, affine=affine, Nfields=nf, dim=dim)
    for ours, k in (("GlobalToLocal", "GlobalToLocal"), ("rowStarts", "rowStartsT"), ("colIds", "colIdsT")):
        a = m.array(ours)
        assert a.size == int(g["size_" + k]), k
        assert digest(a.astype("<i4")) == str(g["sha256_" + k]), k
