"""A batch of independent problems sharded over ranks, one GPU per rank.

The problems of a batch share nothing, so the ranks exchange nothing while
they solve: each rank takes the share that longest-processing-time-first
assignment gives it under a work model, solves that share as one batch on its
own GPU, and the per-problem results are gathered once at the end (one
all-gather of host objects, after the timed solves).  The reference runs one
problem per job, and its ranks split that problem's mesh
(`libs/mesh/meshSetupBoxHex3D.cpp`), so this layer has no counterpart there.
"""


def problem_work(p):
    """Work model of one problem: gathered unknowns x nodes per element x
    right-hand sides (Nd * Np * nrhs), the cost of one CG iteration of its
    operator up to a constant."""
    N = int(p["N"])
    nx = int(p["nx"])
    ny, nz = int(p.get("ny", nx)), int(p.get("nz", nx))
    Nd = (nx * N - 1) * (ny * N - 1) * (nz * N - 1)
    return Nd * (N + 1) ** 3 * int(p.get("nrhs", 1))


def lpt_partition(work, world):
    """Indices of the problems of each rank (ascending within a rank).

    Longest-processing-time first: problems in decreasing work (ties by
    index) each go to the least-loaded rank (ties to the lowest rank).  The
    result is a function of the inputs alone, so every rank computes the
    same partition without communicating.  Its largest load is at most the
    mean load plus the largest single problem."""
    if world < 1:
        raise ValueError("lpt_partition: world must be >= 1")
    load = [0] * world
    share = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        if work[i] < 0:
            raise ValueError("lpt_partition: negative work for problem %d" % i)
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += work[i]
        share[r].append(i)
    return [sorted(s) for s in share]


def solve_sharded(problems, rank, world, solve):
    """Solve this rank's share and gather every rank's results.

    solve(list of problems) -> (list of per-problem results in the same
    order, seconds) runs on this rank's GPU; it is not called for an empty
    share.  Returns (results of all problems in the original order, the
    slowest rank's seconds, this rank's problem indices).  With world > 1 the
    default process group must be up; the one collective is an all-gather of
    host objects after the solves, the same on every rank."""
    problems = list(problems)
    mine = lpt_partition([problem_work(p) for p in problems], world)[rank]
    if mine:
        res, secs = solve([problems[i] for i in mine])
        res = list(res)
        if len(res) != len(mine):
            raise RuntimeError("solve_sharded: %d results for %d problems" % (len(res), len(mine)))
    else:
        res, secs = [], 0.0
    parts = [(dict(zip(mine, res)), float(secs))]
    if world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, (dict(zip(mine, res)), float(secs)))
    merged = {}
    for got, _ in parts:
        for i, v in got.items():
            if i in merged:
                raise RuntimeError("solve_sharded: problem %d solved on two ranks" % i)
            merged[i] = v
    if sorted(merged) != list(range(len(problems))):
        raise RuntimeError("solve_sharded: results of %d of %d problems gathered" % (len(merged), len(problems)))
    return [merged[i] for i in range(len(problems))], max(s for _, s in parts), mine


def batch_solver(tol, maxit, precon="JACOBI", precision="MIXED", warm_iterations=30):
    """A solve function for solve_sharded: the share as one bp.Batch (a short
    warm-up solve, then the timed one); per problem its iterations per
    right-hand side, the largest relative residual and Nd * iterations."""
    def solve(share):
        import numpy as np
        import benchparanumal_b200 as bp
        B = bp.Batch(share, precon=precon, precision=precision)
        try:
            if warm_iterations:
                B.solve(tol=tol, maxit=warm_iterations)
            st, ms = B.solve(tol=tol, maxit=maxit)
            out = []
            for i, p in enumerate(share):
                ks = [k for k in range(B.nsystems) if B.problem[k] == i]
                out.append({"N": int(p["N"]), "n": int(p["nx"]),
                            "iterations": [int(st[k].iterations) for k in ks],
                            "max_relative_residual": max(float(np.sqrt(st[k].rdotr / st[k].rdotr0)) for k in ks),
                            "dof_iterations": int(sum(B.Ngather[k] * st[k].iterations for k in ks))})
            return out, ms / 1e3
        finally:
            del B
    return solve
