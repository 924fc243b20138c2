"""Failure detection on the GPU, in the forms that fault, trap or hang nothing.

* A bounded device-side wait made to run out: bp_test_wait_timeout runs one
  element of the TMA-staged operator through an instantiation that arms a
  slice's mbarrier but never issues its copies.  The wait gives up after its
  short limit, the block drains its own copies (bounded) and leaves, and the
  host reads BP_ERROR_TIMEOUT; the context stays usable.
* Non-finite values injected into host-prepared inputs (right-hand side,
  geometric factors): the device-side breakdown status of the CG
  (p.Ap <= 0, non-finite alpha or residual) comes back as BP_ERROR_NUMERIC from
  bp_solver_solve and bp_batch_solve, FP64 and mixed precision.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("slice_", [0, 3, 5, 7])
def test_withheld_copy_times_out_and_context_survives(gpu, oracle, slice_):
    rc = gpu.lib().bp_test_wait_timeout(slice_)
    assert rc == gpu.BP_ERROR_TIMEOUT, (rc, gpu.lib().bp_last_error())
    assert "gave up" in gpu.lib().bp_last_error().decode()
    # the status was read and cleared; the product kernel runs clean and right
    assert gpu.lib().bp_test_wait_timeout(-1) == gpu.BP_SUCCESS
    om = oracle.Mesh(3, 2, 2, 7, pert=0.1)
    gm = gpu.Mesh(3, 2, 2, N=7, pert=0.1)
    q = 2 * oracle.random(3, om.Ngather) - 1
    dq, dA = gpu.DeviceBuffer.from_host(q), gpu.DeviceBuffer(om.NL)
    gpu.ax_hex3d(gm, dq, dA)
    gpu.finish()
    want = om.ax(q)
    assert np.max(np.abs(dA.download() - want)) <= 1e-12 * np.max(np.abs(want))


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_non_finite_rhs_reports_numeric_error(gpu, precision, bad):
    gm = gpu.Mesh(4, 4, 4, N=4, pert=0.1)
    S = gpu.BP(gm, precon="JACOBI", precision=precision)
    b = S.rhs("RANDOM", 0).download()
    b[17] = bad
    x = gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather))
    with pytest.raises(gpu.BPError, match="breakdown") as e:
        S.solve(x, gpu.DeviceBuffer.from_host(b), tol=1e-8, maxit=300)
    assert e.value.code == gpu.BP_ERROR_NUMERIC
    # the solver still works on a clean right-hand side afterwards
    st, _, _ = S.solve(gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather)), S.rhs("RANDOM", 0), tol=1e-8, maxit=2000)
    assert np.sqrt(st.rdotr / st.rdotr0) <= 1e-8


def test_non_finite_factor_reports_numeric_error(gpu):
    gm = gpu.Mesh(4, 4, 4, N=5, pert=0.1)
    bad = np.array([np.nan])
    # one geometric factor of element 9 becomes NaN (device copy of a host value)
    off = (9 * gm.Np + 40) * 6 + 3
    gpu._check(gpu.lib().bp_memcpy_htod(gm.view.ggeo + 8 * off, bad.ctypes.data, 8, None))
    gpu.finish()
    S = gpu.BP(gm, precon="NONE")
    x = gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather))
    with pytest.raises(gpu.BPError, match="breakdown") as e:
        S.solve(x, S.rhs("RANDOM", 0), tol=1e-8, maxit=300)
    assert e.value.code == gpu.BP_ERROR_NUMERIC


def test_batch_reports_numeric_error_of_one_system(gpu):
    B = gpu.Batch([{"nx": 3, "N": 4, "pert": 0.1, "nrhs": 2, "rhs_seed": 0},
                   {"nx": 4, "N": 3, "pert": 0.1, "nrhs": 1, "rhs_seed": 5}], precon="JACOBI", precision="MIXED")
    xp, bp_ = ctypes.c_void_p(), ctypes.c_void_p()
    gpu._check(gpu.lib().bp_batch_vectors(B._h, 1, ctypes.byref(xp), ctypes.byref(bp_)))
    bad = np.array([np.inf])
    gpu._check(gpu.lib().bp_memcpy_htod(bp_.value + 8 * 10, bad.ctypes.data, 8, None))
    gpu.finish()
    with pytest.raises(gpu.BPError, match="breakdown") as e:
        B.solve(tol=1e-8, maxit=300)
    assert e.value.code == gpu.BP_ERROR_NUMERIC
