"""The allocation-free operator entry point, checked against the allocating one
and against the oracle.

bp_operator_hex3d_noalloc serves callers that cannot call cudaMalloc (their
own pool allocator owns the device memory, or they cannot take the device-wide
synchronisation an allocation implies); it keeps the element-local results in
a fixed array inside the library.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the element-operator tolerance of the parity tests

CASES = [(6, 5, 4, 7, False, 0.1, 1), (8, 8, 8, 4, True, 0.0, 1), (4, 3, 3, 5, False, 0.1, 1),
         (3, 3, 2, 4, False, 0.0, 3)]


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("nx,ny,nz,N,affine,pert,Nf", CASES)
def test_noalloc_operator_matches_allocating_operator_and_oracle(gpu, oracle, nx, ny, nz, N, affine, pert, Nf):
    mesh = gpu.Mesh(nx, ny, nz, N=N, affine=affine, pert=pert, Nfields=Nf)
    om = oracle.Mesh(nx, ny, nz, N, affine=affine, Nfields=Nf, pert=pert)
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
        assert _rel(a, b) <= TOL, call
        assert _rel(a, om.operator(q, bp=6 if Nf == 3 else 5)) <= TOL, call


def test_noalloc_partial_element_list_on_a_user_stream(gpu):
    """A subset of the elements, on a stream the caller created: equal to the
    element operator on the same list into a zeroed E-vector, then the gather."""
    mesh = gpu.Mesh(5, 4, 3, N=5, pert=0.1)
    rng = np.random.default_rng(3)
    sub = np.sort(rng.choice(mesh.E, size=mesh.E // 2, replace=False)).astype(np.int32)
    dsub = gpu.DeviceBuffer.from_host(sub)
    stream = ctypes.c_void_p()
    gpu._check(gpu.lib().bp_stream_create(ctypes.byref(stream)))
    try:
        for call in range(2):
            q = rng.uniform(-1.0, 1.0, mesh.Ngather)
            dq = gpu.DeviceBuffer.from_host(q)
            AqL = gpu.DeviceBuffer(mesh.NL)
            AqL.zero()
            want = gpu.DeviceBuffer(mesh.Ngather)
            gpu.ax_hex3d(mesh, dq, AqL, elementList=dsub.ptr, Nelements=sub.size)
            gpu.ogs_gather(mesh, AqL, want)
            out = gpu.DeviceBuffer(mesh.Ngather)
            gpu.operator_noalloc(mesh, dq, out, stream=stream, elements=dsub, nelements=sub.size)
            gpu._check(gpu.lib().bp_finish(stream))
            assert _rel(out.download(), want.download()) <= TOL, call
    finally:
        gpu.lib().bp_stream_destroy(stream)


def test_noalloc_operator_rejects_meshes_beyond_the_scratch(gpu):
    mesh = gpu.Mesh(14, 14, 14, N=7)            # 14^3 * 8^3 = 1,404,928 local nodes > 2^20
    assert mesh.NL > gpu.NOALLOC_MAX_LOCAL
    dq, out = gpu.DeviceBuffer(mesh.Ngather), gpu.DeviceBuffer(mesh.Ngather)
    with pytest.raises(gpu.BPError, match="scratch maximum"):
        gpu.operator_noalloc(mesh, dq, out)


def test_noalloc_operator_rejects_indices_beyond_nlocal(gpu):
    """Indices at or above Nlocal are found by the device check and reported
    before any launch.  Nlocal is set one element short of the mesh, so every
    array the operator would read stays inside the mesh's own buffers and every
    scratch entry it would touch inside the 8 MiB array either way."""
    mesh = gpu.Mesh(3, 3, 2, N=4)
    Nel = mesh.Np * mesh.Nfields
    short = mesh.NL - Nel
    dq, out = gpu.DeviceBuffer.from_host(np.ones(mesh.Ngather)), gpu.DeviceBuffer(mesh.Ngather)
    with pytest.raises(gpu.BPError, match="exceeds Nlocal"):       # host check: too many elements
        gpu.operator_noalloc(mesh, dq, out, nlocal=short)
    last = gpu.DeviceBuffer.from_host(np.arange(1, mesh.E, dtype=np.int32))   # E-1 ids, the last one E-1
    with pytest.raises(gpu.BPError, match="elementList entry"):
        gpu.operator_noalloc(mesh, dq, out, elements=last, nelements=mesh.E - 1, nlocal=short)
    first = gpu.DeviceBuffer.from_host(np.arange(mesh.E - 1, dtype=np.int32))
    with pytest.raises(gpu.BPError, match="colIds entry"):
        gpu.operator_noalloc(mesh, dq, out, elements=first, nelements=mesh.E - 1, nlocal=short)
    with pytest.raises(gpu.BPError, match="whole number of elements"):
        gpu.operator_noalloc(mesh, dq, out, nlocal=mesh.NL - 1)
    # the entry point still works after the rejected calls
    gpu.operator_noalloc(mesh, dq, out)
