"""The pipelined FP32 over-integrated stiffness kernel (ax_cub_pipe_kernel).

BP3 curved, one field, even Nq: a resident grid loops over element groups with
the next groups' element ids, GlobalToLocal, gathered q and factors in flight.
Checked against the FP64 oracle to FP32 accuracy, against the one-element-per-
slot kernel (BP_CUB_PIPE=0, the same phase code: equal to rounding), on boxes
with a partial last group and with more groups than resident blocks, with an
element list that is a permuted subset, and inside the mixed-precision CG.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _f32_ops(gpu, gm):
    c = gm.cubature()
    nc = gm.E * c.cubNp
    sizes = {"cubwJ": nc, "cubggeo": 6 * nc, "cubD": c.cubNq * c.cubNq, "cubInterp": c.cubNq * gm.Nq,
             "invV": gm.Nq * gm.Nq, "MM": gm.Nq * gm.Nq}
    ops = {}
    for name, n in sizes.items():
        ops[name] = gpu.DeviceBuffer(n, np.float32)
        gpu.convert_f64_f32(getattr(c, name), n, ops[name])
    return ops


def _apply(gpu, gm, ops, dq, dA, elist=None, nel=None):
    d = gpu.AxDesc(3, gm.N, 0, 1)
    v = gm.view
    gpu._check(gpu.lib().bp_ax_cub_hex3d_f32(gpu.ctypes.byref(d), gm.E if nel is None else nel,
                                             v.elementList if elist is None else elist.ptr, v.GlobalToLocal,
                                             ops["cubwJ"].ptr, ops["cubggeo"].ptr, ops["cubD"].ptr,
                                             ops["cubInterp"].ptr, ops["invV"].ptr, ops["MM"].ptr, 1.0, dq.ptr,
                                             dA.ptr, None))


@pytest.mark.parametrize("nx,ny,nz,N", [(3, 2, 2, 7), (5, 5, 5, 7), (10, 10, 10, 7), (4, 3, 3, 5), (3, 3, 2, 3),
                                        (2, 2, 2, 11), (2, 1, 1, 13), (3, 3, 3, 1)])
def test_pipelined_operator_matches_oracle_and_slot_kernel(gpu, oracle, monkeypatch, nx, ny, nz, N):
    # 10^3 at p=7: 334 groups of three elements, more than one wave of resident blocks
    om = oracle.Mesh(nx, ny, nz, N, pert=0.1)
    gm = gpu.Mesh(nx, ny, nz, N=N, pert=0.1)
    ops = _f32_ops(gpu, gm)
    q = (2 * oracle.random(8, om.Ngather) - 1).astype(np.float32)
    dq = gpu.DeviceBuffer.from_host(q)
    out = {}
    for pipe in ("1", "0"):
        monkeypatch.setenv("BP_CUB_PIPE", pipe)
        dA = gpu.DeviceBuffer.from_host(np.full(om.NL, np.nan, np.float32))
        _apply(gpu, gm, ops, dq, dA)
        out[pipe] = dA.download()
    monkeypatch.delenv("BP_CUB_PIPE")
    assert not np.any(np.isnan(out["1"]))   # every element's nodes written
    want = om.ax(q.astype(np.float64), 1.0, 3)
    assert _rel(out["1"].astype(np.float64), want) < 2e-5
    assert _rel(out["1"], out["0"]) < 1e-6


def test_pipelined_operator_on_a_permuted_subset(gpu, oracle):
    # a partial element list in shuffled order: exactly the listed elements are written
    om = oracle.Mesh(6, 5, 4, 7, pert=0.1)
    gm = gpu.Mesh(6, 5, 4, N=7, pert=0.1)
    ops = _f32_ops(gpu, gm)
    q = (2 * oracle.random(9, om.Ngather) - 1).astype(np.float32)
    dq = gpu.DeviceBuffer.from_host(q)
    rng = np.random.default_rng(3)
    sub = rng.permutation(gm.E)[: gm.E // 2 + 1].astype(np.int32)   # an odd count: a partial last group
    dl = gpu.DeviceBuffer.from_host(sub)
    dA = gpu.DeviceBuffer.from_host(np.full(om.NL, np.nan, np.float32))
    _apply(gpu, gm, ops, dq, dA, elist=dl, nel=sub.size)
    got = dA.download().reshape(gm.E, gm.Np)
    want = om.ax(q.astype(np.float64), 1.0, 3).reshape(gm.E, gm.Np)
    listed = np.zeros(gm.E, bool)
    listed[sub] = True
    assert np.all(np.isnan(got[~listed]))
    assert _rel(got[listed].astype(np.float64), want[listed]) < 2e-5


def test_mixed_bp3_with_pipelined_kernel_matches_slot_kernel(gpu, oracle, monkeypatch):
    # the fused p.Ap partials (one per block over all its groups) drive alpha
    res = {}
    om = oracle.Mesh(6, 6, 5, 7, pert=0.1)
    _, b_o = om.rhs_random(0)
    for pipe in ("1", "0"):
        monkeypatch.setenv("BP_CUB_PIPE", pipe)
        gm = gpu.Mesh(6, 6, 5, N=7, pert=0.1)
        S = gpu.BP(gm, bp=3, precon="JACOBI", precision="MIXED")
        x = gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather))
        st, _, _ = S.solve(x, gpu.DeviceBuffer.from_host(b_o), tol=1e-8, maxit=5000)
        res[pipe] = (st.iterations, x.download())
    monkeypatch.delenv("BP_CUB_PIPE")
    for pipe in ("1", "0"):
        assert np.linalg.norm(b_o - om.operator(res[pipe][1], bp=3)) <= 1.0001e-8 * np.linalg.norm(b_o)
    assert abs(res["1"][0] - res["0"][0]) <= 3
    assert _rel(res["1"][1], res["0"][1]) < 1e-6
