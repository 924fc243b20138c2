"""Programmatic dependent launch of the CG iteration kernels.

With PDL a kernel may be scheduled while its predecessor finishes and waits in
griddepcontrol.wait for the predecessor's results; without it the kernels run
one after the other.  Both orders must give the same numbers: FP64 and packed
mixed-precision solves run here with PDL on (the default) and in a child process
with BP_PDL=0 (read once per process), and their residual histories, iteration
counts and solutions must agree bit for bit.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, %r)
import benchparanumal_b200 as bp
bp.platform_init(0)
out = {}
gm = bp.Mesh(4, 3, 3, N=7, pert=0.1)
S = bp.BP(gm, precon="JACOBI")
x = bp.DeviceBuffer.from_host(np.zeros(gm.Ngather))
st, hr, ha = S.solve(x, S.rhs("RANDOM", 0), tol=0.0, maxit=60)
out["fp64"] = [float(v) for v in hr] + [float(v) for v in x.download()[:64]]
B = bp.Batch([{"nx": 4, "ny": 3, "nz": 3, "N": 7, "pert": 0.1, "pert_seed": 1, "nrhs": 4, "rhs_seed": 0}],
             precon="JACOBI", precision="MIXED")
stats, _ = B.solve(tol=1e-8, maxit=3000)
out["mixed_it"] = [int(s.iterations) for s in stats]
out["mixed_x"] = [float(v) for v in B.vectors(0)[0][:64]]
print(json.dumps(out))
""" % ROOT


def _run(pdl):
    # one operator form in both processes (the autotuner's timing could pick
    # different forms, and forms differ in rounding)
    env = dict(os.environ, BP_PDL=pdl, BP_AX_VARIANT="tma")
    r = subprocess.run([sys.executable, "-c", CHILD], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_pdl_and_serial_launches_give_the_same_solves():
    on, off = _run("1"), _run("0")
    assert on["mixed_it"] == off["mixed_it"]
    np.testing.assert_array_equal(np.array(on["fp64"]), np.array(off["fp64"]))
    np.testing.assert_array_equal(np.array(on["mixed_x"]), np.array(off["mixed_x"]))
