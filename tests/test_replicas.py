"""The multi-GPU path of bench.py is replicas only: every rank solves its own
copy and the timing is the slowest rank's.  The host logic of that path (the
max over ranks, the barrier) runs here on two gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        bench.barrier(world)
        out[rank] = bench.max_over_ranks(1.5 + rank, world)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        assert dict(out) == {0: 2.5, 1: 2.5}
