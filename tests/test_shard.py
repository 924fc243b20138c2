"""The batch sharded over ranks (benchparanumal_b200/shard.py): the partition
and the final result gather, on the CPU.  Two gloo ranks stand in for two
GPUs; the solve function is a stand-in that needs no GPU."""
import os
import socket

import pytest

from benchparanumal_b200 import uneven_problems
from benchparanumal_b200.shard import lpt_partition, problem_work, solve_sharded


def test_problem_work_model():
    p = {"nx": 8, "N": 3, "nrhs": 4}
    assert problem_work(p) == 23 ** 3 * 4 ** 3 * 4
    assert problem_work({"nx": 2, "ny": 3, "nz": 4, "N": 2}) == 3 * 5 * 7 * 27


@pytest.mark.parametrize("world", [1, 2, 3, 8, 70])
def test_lpt_partition_covers_each_problem_once(world):
    work = [problem_work(p) for p in uneven_problems()]
    share = lpt_partition(work, world)
    assert len(share) == world
    flat = sorted(i for s in share for i in s)
    assert flat == list(range(len(work)))
    assert all(s == sorted(s) for s in share)
    loads = [sum(work[i] for i in s) for s in share]
    # the LPT bound: no rank above the mean load plus the largest problem
    assert max(loads) <= sum(work) / world + max(work)
    if world > len(work):
        assert sum(1 for s in share if not s) == world - len(work)


def test_lpt_partition_is_deterministic_and_greedy():
    work = [5, 7, 7, 3, 2, 2, 9]
    # decreasing work, ties by index: 6(9) 1(7) 2(7) 0(5) 3(3) 4(2) 5(2)
    # loads after each: [9,0] [9,7] [9,14] [14,14] [17,14] [17,16] [17,18]
    assert lpt_partition(work, 2) == [[0, 3, 6], [1, 2, 4, 5]]
    assert lpt_partition(work, 2) == lpt_partition(list(work), 2)
    assert lpt_partition([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        lpt_partition(work, 0)
    with pytest.raises(ValueError):
        lpt_partition([1, -1], 2)


def _fake_solve(rank):
    """Per problem a result computed from the problem alone; seconds by rank."""
    def solve(share):
        return [{"N": p["N"], "n": p["nx"], "iterations": [p["N"] * p["nx"]] * p["nrhs"]} for p in share], 1.0 + rank
    return solve


def test_solve_sharded_one_rank_keeps_order():
    probs = uneven_problems(count=10)
    res, secs, mine = solve_sharded(probs, 0, 1, _fake_solve(0))
    assert mine == list(range(10)) and secs == 1.0
    assert [r["N"] for r in res] == [p["N"] for p in probs]


def test_solve_sharded_rejects_a_short_result():
    probs = uneven_problems(count=3)
    with pytest.raises(RuntimeError):
        solve_sharded(probs, 0, 1, lambda share: (share[:-1], 0.0))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        probs = uneven_problems(count=12)
        calls = []

        def solve(share):
            calls.append(len(share))
            return _fake_solve(rank)(share)

        res, secs, mine = solve_sharded(probs, rank, world, solve)
        out[rank] = (res, secs, mine, calls)
    finally:
        dist.destroy_process_group()


def test_solve_sharded_two_gloo_ranks():
    pytest.importorskip("torch")
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        got = dict(out)
    probs = uneven_problems(count=12)
    serial, _, _ = solve_sharded(probs, 0, 1, _fake_solve(0))
    share = lpt_partition([problem_work(p) for p in probs], 2)
    for rank in (0, 1):
        res, secs, mine, calls = got[rank]
        assert res == serial            # every rank holds every problem's result, in order
        assert secs == 2.0              # the slowest rank's seconds
        assert mine == share[rank] and calls == [len(share[rank])]
