"""A batch sharded over ranks solves each problem as the whole batch does:
the problems are independent, so every share, solved alone on the GPU, gives
the same iterations per right-hand side as the whole batch."""
import pytest

from benchparanumal_b200.shard import batch_solver, lpt_partition, problem_work, solve_sharded

pytestmark = pytest.mark.gpu


def test_shares_solve_like_the_whole_batch(gpu):
    probs = gpu.uneven_problems(count=6, pmin=3, pmax=6, nmin=2, nmax=6)
    solve = batch_solver(1e-8, 4000)
    whole, secs, mine = solve_sharded(probs, 0, 1, solve)
    assert mine == list(range(len(probs))) and secs > 0
    for r in whole:
        assert r["max_relative_residual"] <= 1e-8
        assert len(r["iterations"]) == 4 and min(r["iterations"]) > 0
    share = lpt_partition([problem_work(p) for p in probs], 2)
    assert all(share)
    for s in share:
        res, _ = solve([probs[i] for i in s])
        for i, got in zip(s, res):
            assert got["iterations"] == whole[i]["iterations"]
            assert got["dof_iterations"] == whole[i]["dof_iterations"]
            assert got["max_relative_residual"] <= 1e-8
