"""The "-o" output of the BP drivers (BP/BP5/src/bp5Run.cpp:220-238): the
solution scattered to the element nodes, written by bp_mesh_write_vtu as a VTK
XML unstructured grid (libs/mesh/meshPlotFields3D.cpp:31-113) of the element
nodes and six tetrahedra per node sub-cube.
"""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _read_vtu(path):
    piece = ET.parse(path).getroot().find("UnstructuredGrid/Piece")
    arrays = {}
    for da in piece.iter("DataArray"):
        name = da.get("Name") or "Points"
        dt = np.int64 if da.get("type") == "Int32" else np.float64
        arrays[name] = (np.array(da.text.split(), dtype=dt), int(da.get("NumberOfComponents", "1")))
    return int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells")), arrays


def _nodes(gm):
    """Element node coordinates [E*Np, 3] by the trilinear vertex map at the GLL nodes."""
    z = gm.array("gllz")
    t, s, r = np.meshgrid(z, z, z, indexing="ij")
    shape = np.stack([(1 - r) * (1 - s) * (1 - t), (1 + r) * (1 - s) * (1 - t), (1 + r) * (1 + s) * (1 - t),
                      (1 - r) * (1 + s) * (1 - t), (1 - r) * (1 - s) * (1 + t), (1 + r) * (1 - s) * (1 + t),
                      (1 + r) * (1 + s) * (1 + t), (1 - r) * (1 + s) * (1 + t)]).reshape(8, -1) / 8
    xyz = [gm.array(n).reshape(gm.E, 8) @ shape for n in ("EX", "EY", "EZ")]
    return np.stack([c.reshape(-1) for c in xyz], axis=1)


def _tet_volumes(pts, conn):
    p = pts[conn.reshape(-1, 4)]
    return np.linalg.det(np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]], axis=1)) / 6


@pytest.mark.parametrize("N,Nfields,pert", [(1, 1, 0.0), (3, 1, 0.1), (5, 3, 0.0)])
def test_write_vtu_points_fields_cells(gpu, tmp_path, N, Nfields, pert):
    gm = gpu.Mesh(2, 3, 2, N=N, Nfields=Nfields, pert=pert)
    rng = np.random.default_rng(3)
    xL = rng.standard_normal(gm.NL)
    path = tmp_path / "field_0000.vtu"
    gm.write_vtu(xL, path)
    npts, ncells, a = _read_vtu(path)
    assert npts == gm.E * gm.Np and ncells == 6 * gm.E * N ** 3
    pts = a["Points"][0].reshape(-1, 3)
    ref = _nodes(gm)
    assert np.abs(pts - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())
    f, nc = a["Fields"]
    assert nc == Nfields
    want = xL.reshape(gm.E, Nfields, gm.Np).transpose(0, 2, 1).reshape(-1)
    assert np.allclose(f, want, rtol=1e-5, atol=1e-5)
    conn = a["connectivity"][0]
    assert conn.size == 4 * ncells and conn.min() >= 0 and conn.max() < npts
    assert np.array_equal(a["offsets"][0], 4 * np.arange(1, ncells + 1))
    assert np.all(a["types"][0] == 10)
    # every tetrahedron positively oriented; on the unperturbed box they tile it
    vol = _tet_volumes(ref, conn)
    assert vol.min() > 0
    if pert == 0.0:
        lo, hi = ref.min(axis=0), ref.max(axis=0)
        assert abs(vol.sum() - np.prod(hi - lo)) < 1e-10 * np.prod(hi - lo)


def test_write_vtu_bad_args(gpu, tmp_path):
    gm = gpu.Mesh(2, 2, 2, N=2)
    with pytest.raises(ValueError):
        gm.write_vtu(np.zeros(3), tmp_path / "x.vtu")
    with pytest.raises(gpu.BPError):
        gm.write_vtu(np.zeros(gm.NL), tmp_path / "missing_dir" / "x.vtu")


@pytest.mark.parametrize("k", [5, 3])
def test_driver_output_file(gpu, capfd, tmp_path, k):
    """BPk -o name writes name_0000.vtu with the scattered solution: continuous
    across element faces and zero on the Dirichlet boundary."""
    name = str(tmp_path / "sol")
    args = ["-nx", "3", "-ny", "2", "-nz", "2", "-p", "3", "-it", "30", "-pt", "0.1", "-o", name]
    assert gpu.driver_main("BP%d" % k, args) == 0
    capfd.readouterr()
    npts, ncells, a = _read_vtu(name + "_0000.vtu")
    gm = gpu.Mesh(3, 2, 2, N=3, pert=0.1)
    assert npts == gm.E * gm.Np and ncells == 6 * gm.E * 27
    f = a["Fields"][0]
    g2l = gm.array("GlobalToLocal")
    rows, cols = gm.array("rowStarts"), gm.array("colIds")
    assert np.all(f[g2l < 0] == 0) and np.abs(f).max() > 0
    for r in range(gm.Ngather):
        vals = f[cols[rows[r]:rows[r + 1]]]
        assert np.all(vals == vals[0])
