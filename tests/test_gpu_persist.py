"""One CG step of a packed group as one cooperative kernel (bp_cg_persist.cuh).

Small packed groups run each step as a single resident grid with grid barriers
between the direction, operator, alpha and gather-update phases.  Forced on
(BP_PERSIST=1) and off (0) on the same small problems -- the line form (odd
Nq) and the TMA form (Nq = 8) of the operator -- both must reach the FP64
residual 1e-8 (checked with the oracle's operator) in the same iteration
counts (within 3: the sums are grouped differently), with one kernel per step
instead of four.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROBLEMS = [{"nx": 6, "ny": 5, "nz": 4, "N": 4, "pert": 0.1, "pert_seed": 3, "nrhs": 4, "rhs_seed": 0},
            {"nx": 4, "ny": 4, "nz": 3, "N": 7, "pert": 0.1, "pert_seed": 1, "nrhs": 4, "rhs_seed": 4},
            {"nx": 5, "ny": 4, "nz": 4, "N": 3, "affine": True, "nrhs": 3, "rhs_seed": 8}]


def _solve(gpu, flag):
    os.environ["BP_PERSIST"] = flag
    try:
        B = gpu.Batch(PROBLEMS, precon="JACOBI", precision="MIXED")
        stats, _ = B.solve(tol=1e-8, maxit=3000)
        return B, stats
    finally:
        os.environ.pop("BP_PERSIST", None)


def test_persistent_step_matches_graph_step(gpu, oracle):
    Bp, sp = _solve(gpu, "1")
    Bg, sg = _solve(gpu, "0")
    assert len(sp) == len(sg) == 11
    assert all(abs(a.iterations - b.iterations) <= 3 for a, b in zip(sp, sg))
    launches_p = sum(s.kernel_launches for s in sp)
    launches_g = sum(s.kernel_launches for s in sg)
    assert launches_p < launches_g
    k = 0
    for P in PROBLEMS:
        om = oracle.Mesh(P["nx"], P["ny"], P["nz"], P["N"], affine=P.get("affine", False),
                         pert=P.get("pert", 0.0), pert_seed=P.get("pert_seed", 1))
        for j in range(P["nrhs"]):
            _, b_o = om.rhs_random(P["rhs_seed"] + j)
            for B in (Bp, Bg):
                x = B.vectors(k)[0]
                assert np.linalg.norm(b_o - om.operator(x)) <= 1.0001e-8 * np.linalg.norm(b_o)
            k += 1


def test_persistent_step_on_uneven_small_problems(gpu, oracle):
    probs = [{"nx": 3 + i % 3, "ny": 3, "nz": 2 + i % 2, "N": 3 + i, "pert": 0.1, "pert_seed": 10 + i, "nrhs": 4,
              "rhs_seed": 100 + 4 * i} for i in range(8)]   # Nq 4..11: line and TMA forms
    os.environ["BP_PERSIST"] = "1"
    try:
        B = gpu.Batch(probs, precon="JACOBI", precision="MIXED")
        stats, _ = B.solve(tol=1e-8, maxit=5000)
    finally:
        os.environ.pop("BP_PERSIST", None)
    k = 0
    for P in probs:
        om = oracle.Mesh(P["nx"], P["ny"], P["nz"], P["N"], pert=P["pert"], pert_seed=P["pert_seed"])
        for j in range(4):
            _, b_o = om.rhs_random(P["rhs_seed"] + j)
            x = B.vectors(k)[0]
            assert np.linalg.norm(b_o - om.operator(x)) <= 1.0001e-8 * np.linalg.norm(b_o), (P, j)
            k += 1
