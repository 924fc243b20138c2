"""The allocation-free operator entry point, checked against the allocating one.

bp_operator_hex3d_noalloc serves callers that cannot call cudaMalloc (their
own pool allocator owns the device memory, or they cannot take the device-wide
synchronisation an allocation implies); it keeps the element-local results in
a fixed array inside the library.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the element-operator tolerance of the parity tests


@pytest.mark.parametrize("nx,ny,nz,N,affine,pert,Nf", [(6, 5, 4, 7, False, 0.1, 1), (8, 8, 8, 4, True, 0.0, 1),
                                                        (4, 3, 3, 5, False, 0.1, 1), (3, 3, 2, 4, False, 0.0, 3)])
def test_noalloc_operator_matches_allocating_operator(gpu, nx, ny, nz, N, affine, pert, Nf):
    mesh = gpu.Mesh(nx, ny, nz, N=N, affine=affine, pert=pert, Nfields=Nf)
    assert mesh.NL <= gpu.NOALLOC_MAX_LOCAL
    S = gpu.BP(mesh)
    rng = np.random.default_rng(7)
    for call in range(2):                       # two calls in a row share the scratch array
        q = rng.uniform(-1.0, 1.0, mesh.Ngather)
        dq = gpu.DeviceBuffer.from_host(q)
        ref, out = gpu.DeviceBuffer(mesh.Ngather), gpu.DeviceBuffer(mesh.Ngather)
        S.operator(dq, ref)
        gpu.operator_noalloc(mesh, dq, out)
        a, b = out.download(), ref.download()
        assert np.max(np.abs(a - b)) <= TOL * np.max(np.abs(b)), call


def test_noalloc_operator_rejects_meshes_beyond_the_scratch(gpu):
    mesh = gpu.Mesh(14, 14, 14, N=7)            # 14^3 * 8^3 = 1,404,928 local nodes > 2^20
    assert mesh.NL > gpu.NOALLOC_MAX_LOCAL
    dq, out = gpu.DeviceBuffer(mesh.Ngather), gpu.DeviceBuffer(mesh.Ngather)
    with pytest.raises(gpu.BPError, match="scratch maximum"):
        gpu.operator_noalloc(mesh, dq, out)
