"""The register-blocked packed FP32 operator (BP_AX_VARIANT=rb).

One lane of four k-pencils per thread, mirrored rows and columns of D taken
from its antisymmetry (exact for the GLL matrix, to an FP32 ulp for the
computed one).  Each lane must equal the FP64 oracle's operator to
FP32 accuracy and the packed TMA form to 1e-6; a mixed batch solved with it
must reach 1e-8 in FP64 with the iteration counts of the default form.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _ops(gpu, gm):
    v = gm.view
    ng = gm.E * gm.Np
    ops = {"wJ": gpu.DeviceBuffer(ng, np.float32), "ggeo": gpu.DeviceBuffer(6 * ng, np.float32),
           "gllw": gpu.DeviceBuffer(gm.Nq, np.float32), "D": gpu.DeviceBuffer(gm.Nq * gm.Nq, np.float32)}
    for name, n in (("wJ", ng), ("ggeo", 6 * ng), ("gllw", gm.Nq), ("D", gm.Nq * gm.Nq)):
        gpu.convert_f64_f32(getattr(v, name), n, ops[name])
    return ops


def test_gll_differentiation_matrix_is_antisymmetric(gpu):
    # The property the form relies on: the exact GLL D is antisymmetric, the
    # computed one to rounding (FP64 1e-14 absolute; its FP32 copy to an ulp or
    # two), so the mirrored rows the form uses differ from the given ones far
    # below the FP32 operator's accuracy.
    for N in range(1, 16):
        gm = gpu.Mesh(1, 1, 1, N=N)
        D32 = gm.array("D").astype(np.float32).reshape(N + 1, N + 1)
        assert np.max(np.abs(D32[::-1, ::-1] + D32)) <= 4 * np.finfo(np.float32).eps * np.max(np.abs(D32)), N


@pytest.mark.parametrize("form", ["rb"])
@pytest.mark.parametrize("nx,ny,nz,pert", [(3, 2, 2, 0.1), (2, 2, 2, 0.0), (5, 3, 2, 0.2), (2, 1, 1, 0.0)])
def test_packed_form_matches_oracle_and_tma_form(gpu, oracle, monkeypatch, form, nx, ny, nz, pert):
    N = 7
    om = oracle.Mesh(nx, ny, nz, N, pert=pert)
    gm = gpu.Mesh(nx, ny, nz, N=N, pert=pert)
    ops = _ops(gpu, gm)
    Q = np.stack([2 * oracle.random(40 + k, gm.Ngather) - 1 for k in range(4)], axis=1).astype(np.float32)
    dq = gpu.DeviceBuffer.from_host(np.ascontiguousarray(Q).ravel())
    out = {}
    for f in (form, "tma"):
        monkeypatch.setenv("BP_AX_VARIANT", f)
        dA = gpu.DeviceBuffer.from_host(np.full(gm.NL * 4, np.nan, np.float32))
        gpu.ax_hex3d_f32_multi(gm, 4, dq, dA, ops)
        out[f] = dA.download().reshape(gm.NL, 4)
    monkeypatch.delenv("BP_AX_VARIANT")
    assert not np.any(np.isnan(out[form]))   # every entry written, masked nodes included
    for k in range(4):
        want = om.ax(Q[:, k].astype(np.float64))
        assert rel(out[form][:, k].astype(np.float64), want) <= 2e-6
        assert rel(out[form][:, k], out["tma"][:, k]) <= 1e-6


@pytest.mark.parametrize("form", ["rb"])
def test_packed_form_in_mixed_batch(gpu, oracle, monkeypatch, form):
    res = {}
    for f in (form, "tma"):
        monkeypatch.setenv("BP_AX_VARIANT", f)
        B = gpu.Batch([{"nx": 4, "ny": 4, "nz": 3, "N": 7, "pert": 0.1, "pert_seed": 1, "nrhs": 4, "rhs_seed": 0}],
                      precon="JACOBI", precision="MIXED")
        stats, _ = B.solve(tol=1e-8, maxit=3000)
        res[f] = ([s.iterations for s in stats], [B.vectors(k)[0] for k in range(4)])
    monkeypatch.delenv("BP_AX_VARIANT")
    om = oracle.Mesh(4, 4, 3, 7, pert=0.1)
    for k in range(4):
        _, b_o = om.rhs_random(k)
        x = res[form][1][k]
        assert np.linalg.norm(b_o - om.operator(x)) <= 1.0001e-8 * np.linalg.norm(b_o)
    assert all(abs(a - b) <= 3 for a, b in zip(res[form][0], res["tma"][0]))
