"""Batched solves (bp_batch_*): many problems of uneven degree and size with
several right-hand sides each, solved together, against the single-problem
solver and the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROBLEMS = [
    {"nx": 3, "N": 3, "pert": 0.1, "pert_seed": 100, "nrhs": 2, "rhs_seed": 1000},
    {"nx": 4, "N": 5, "pert": 0.1, "pert_seed": 101, "nrhs": 3, "rhs_seed": 1002},
    {"nx": 2, "N": 7, "pert": 0.1, "pert_seed": 102, "nrhs": 1, "rhs_seed": 1005},
    {"nx": 3, "N": 10, "pert": 0.1, "pert_seed": 103, "nrhs": 3, "rhs_seed": 1006},
    {"nx": 2, "N": 7, "pert": 0.1, "pert_seed": 104, "nrhs": 4, "rhs_seed": 1009},
]
# In a mixed batch the right-hand sides of a problem run as packed groups:
# problem 0 as two lanes, problems 1 and 3 as four lanes with one idle,
# problem 4 as four lanes; problem 2 (one right-hand side) is a standalone
# system.


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def test_batch_fp64_matches_single_solver(gpu):
    B = gpu.Batch(PROBLEMS, precon="JACOBI", precision="FP64")
    assert B.nsystems == sum(p["nrhs"] for p in PROBLEMS)
    stats, ms = B.solve(tol=1e-8, maxit=3000)
    assert ms > 0
    sysno = 0
    for j, p in enumerate(PROBLEMS):
        gm = gpu.Mesh(p["nx"], N=p["N"], pert=p["pert"], pert_seed=p["pert_seed"])
        S = gpu.BP(gm, precon="JACOBI")
        for k in range(p["nrhs"]):
            assert B.problem[sysno] == j and B.Ngather[sysno] == gm.Ngather
            b = S.rhs("RANDOM", p["rhs_seed"] + k)
            x = gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather))
            st, _, _ = S.solve(x, b, tol=1e-8, maxit=3000)
            xb, bb = B.vectors(sysno)
            # the same kernels in the same order: the same iterations and solution
            np.testing.assert_array_equal(bb, S.rhs("RANDOM", p["rhs_seed"] + k).download())
            assert stats[sysno].iterations == st.iterations
            assert _rel(xb, x.download()) < 1e-13
            assert np.sqrt(stats[sysno].rdotr / stats[sysno].rdotr0) <= 1e-8
            sysno += 1


def test_batch_mixed_reaches_tolerance_against_oracle(gpu, oracle):
    B = gpu.Batch(PROBLEMS, precon="JACOBI", precision="MIXED")
    stats, _ = B.solve(tol=1e-8, maxit=5000)
    for s in range(B.nsystems):
        p = PROBLEMS[B.problem[s]]
        k = s - sum(PROBLEMS[i]["nrhs"] for i in range(B.problem[s]))
        om = oracle.Mesh(p["nx"], p["nx"], p["nx"], p["N"], pert=p["pert"], pert_seed=p["pert_seed"])
        f_o, b_o = om.rhs_random(p["rhs_seed"] + k)
        xb, bb = B.vectors(s)
        assert _rel(bb, b_o) < 1e-13
        # FP64 residual of the returned solution by the oracle's operator
        r = b_o - om.operator(xb)
        assert np.linalg.norm(r) <= 1.0001e-8 * np.linalg.norm(b_o)
        assert np.sqrt(stats[s].rdotr / stats[s].rdotr0) <= 1e-8
        x_o, _, it_o, _, _ = om.cg(b_o, 1.0, 1e-10, 5000, precon=True)
        assert _rel(xb, x_o) < 1e-5
        assert stats[s].iterations <= 1.25 * it_o + 20


def test_batch_bad_arguments(gpu):
    with pytest.raises(gpu.BPError):
        gpu.Batch([{"nx": 2, "N": 3, "nrhs": 0}])
    with pytest.raises(gpu.BPError):
        gpu.Batch([{"nx": 2, "N": 3, "nrhs": 1}], bp=6)
    B = gpu.Batch([{"nx": 2, "N": 3, "nrhs": 1}], precision="MIXED")
    with pytest.raises(gpu.BPError):
        B.solve(tol=0.0)   # a mixed batch needs a tolerance


def test_batch_splits_and_other_problems(gpu, oracle):
    # six right-hand sides split into a four-lane and a two-lane group; a BP3
    # batch runs standalone over-integrated systems
    B = gpu.Batch([{"nx": 2, "N": 5, "pert": 0.1, "pert_seed": 7, "nrhs": 6, "rhs_seed": 50}], precision="MIXED")
    stats, _ = B.solve(tol=1e-8, maxit=3000)
    om = oracle.Mesh(2, 2, 2, 5, pert=0.1, pert_seed=7)
    for s in range(6):
        xb, bb = B.vectors(s)
        _, b_o = om.rhs_random(50 + s)
        np.testing.assert_allclose(bb, b_o, rtol=0, atol=1e-13 * np.max(np.abs(b_o)))
        assert np.linalg.norm(b_o - om.operator(xb)) <= 1.0001e-8 * np.linalg.norm(b_o)
    B3 = gpu.Batch([{"nx": 2, "N": 4, "pert": 0.1, "pert_seed": 8, "nrhs": 2, "rhs_seed": 60},
                    {"nx": 3, "N": 3, "pert": 0.1, "pert_seed": 9, "nrhs": 1, "rhs_seed": 62}], bp=3,
                   precision="MIXED")
    stats3, _ = B3.solve(tol=1e-8, maxit=3000)
    for s in range(3):
        p = [(2, 4, 8, 60), (2, 4, 8, 61), (3, 3, 9, 62)][s]
        om3 = oracle.Mesh(p[0], p[0], p[0], p[1], pert=0.1, pert_seed=p[2])
        xb, _ = B3.vectors(s)
        _, b_o = om3.rhs_random(p[3])
        assert np.linalg.norm(b_o - om3.operator(xb, 1.0, 3)) <= 1.0001e-8 * np.linalg.norm(b_o)


def test_driver_batched_rhs(gpu, capfd):
    assert gpu.driver_main("BP5", ["-nx", "4", "-ny", "4", "-nz", "4", "-p", "5", "-pt", "0.1", "-f", "RANDOM",
                                   "-pc", "JACOBI", "-fp", "MIXED", "-tol", "1e-8", "-it", "3000", "-nr", "4"]) == 0
    out = capfd.readouterr().out
    line = [l for l in out.splitlines() if l.startswith("BP5: N= 5")][0]
    assert "DOFs=6859," in line and line.endswith("Element=Hex ")
    extra = [l for l in out.splitlines() if l.startswith("BP5 extra: right-hand sides=4 solved together")][0]
    res = [float(v) for v in extra.split("relative residuals:")[1].split(",")[0].split()]
    assert len(res) == 4 and max(res) <= 1.0001e-8


def test_batch_more_units_than_streams(gpu):
    # 40 problems of uneven degree and size (the C5 generator at small sizes) with
    # 2-4 right-hand sides: more units than the 16 streams of the pool, so units
    # are started as others retire.  Every system reaches the tolerance by its own
    # FP64 residual, and the FP64 batch gives each system exactly what a single
    # solve gives it.
    probs = gpu.uneven_problems(count=40, seed=5, nrhs=3, pmin=2, pmax=8, nmin=2, nmax=5)
    probs = [dict(p, nrhs=2 + i % 3) for i, p in enumerate(probs)]
    B = gpu.Batch(probs, precon="JACOBI", precision="MIXED")
    assert B.nsystems == sum(p["nrhs"] for p in probs)
    stats, _ = B.solve(tol=1e-8, maxit=5000)
    stats2, _ = B.solve(tol=1e-8, maxit=5000)   # a second solve on the same batch
    for s in range(B.nsystems):
        assert np.sqrt(stats[s].rdotr / stats[s].rdotr0) <= 1e-8
        assert stats2[s].iterations == stats[s].iterations
    B64 = gpu.Batch(probs[:20], precon="JACOBI", precision="FP64")
    st64, _ = B64.solve(tol=1e-8, maxit=5000)
    sysno = 0
    for j, p in enumerate(probs[:20]):
        gm = gpu.Mesh(p["nx"], N=p["N"], pert=p["pert"], pert_seed=p["pert_seed"])
        S = gpu.BP(gm, precon="JACOBI")
        for k in range(p["nrhs"]):
            b = S.rhs("RANDOM", p["rhs_seed"] + k)
            x = gpu.DeviceBuffer.from_host(np.zeros(gm.Ngather))
            st, _, _ = S.solve(x, b, tol=1e-8, maxit=5000)
            xb, _ = B64.vectors(sysno)
            assert st64[sysno].iterations == st.iterations
            assert _rel(xb, x.download()) < 1e-13
            sysno += 1


def test_batch_affine_problems(gpu, oracle):
    # affine meshes (per-element factors) in a mixed batch: four packed lanes on an
    # even and an odd degree, each system to the tolerance by the oracle's operator
    probs = [{"nx": 3, "N": 4, "nrhs": 4, "rhs_seed": 70, "affine": True},
             {"nx": 2, "N": 7, "nrhs": 3, "rhs_seed": 80, "affine": True}]
    B = gpu.Batch(probs, precon="JACOBI", precision="MIXED")
    stats, _ = B.solve(tol=1e-8, maxit=3000)
    s = 0
    for p in probs:
        om = oracle.Mesh(p["nx"], p["nx"], p["nx"], p["N"], affine=True)
        for k in range(p["nrhs"]):
            xb, bb = B.vectors(s)
            _, b_o = om.rhs_random(p["rhs_seed"] + k)
            assert _rel(bb, b_o) < 1e-13
            assert np.linalg.norm(b_o - om.operator(xb)) <= 1.0001e-8 * np.linalg.norm(b_o)
            s += 1

def test_driver_batched_affine(gpu, capfd):
    assert gpu.driver_main("BP5", ["-nx", "4", "-ny", "4", "-nz", "4", "-p", "4", "-a", "-f", "RANDOM", "-pc", "JACOBI",
                                   "-fp", "MIXED", "-tol", "1e-8", "-it", "3000", "-nr", "4"]) == 0
    out = capfd.readouterr().out
    line = [l for l in out.splitlines() if l.startswith("BP5: N= 4")][0]
    assert line.endswith("Element=Hex, Affine ")


def test_batch_iteration_cap(gpu):
    # a cap below convergence: every lane stops at exactly maxit (mid-chunk for the
    # ten-iteration graphs), with its residual replaced by the FP64 one, and the
    # batch returns; a second solve gives the same counts
    probs = [{"nx": 4, "N": 6, "pert": 0.1, "pert_seed": 3, "nrhs": 4, "rhs_seed": 90},
             {"nx": 3, "N": 5, "pert": 0.1, "pert_seed": 4, "nrhs": 1, "rhs_seed": 95}]
    for prec in ("MIXED", "FP64"):
        B = gpu.Batch(probs, precon="JACOBI", precision=prec)
        stats, _ = B.solve(tol=1e-8, maxit=15)
        assert all(s.iterations == 15 for s in stats)
        assert all(np.sqrt(s.rdotr / s.rdotr0) > 1e-8 for s in stats)
        stats2, _ = B.solve(tol=1e-8, maxit=15)
        assert [s.iterations for s in stats2] == [s.iterations for s in stats]
