"""The N > 1 path of bench.py on CPU: two gloo ranks, each timing its own
replica; the job's time is the maximum over ranks and its value the sum of
all replicas' cell updates over that time."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [10.0 + rank, 3.0 * (world - rank)]  # each rank's own timings
        out[rank] = bench.max_over_ranks(ms)
        torch.distributed.barrier()
    finally:
        torch.distributed.destroy_process_group()


def test_two_ranks_take_the_max_time():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == [11.0, 6.0]


def test_replicas_value_counts_every_rank():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    # 2 replicas of 1e6 cells, 10 steps each, slowest rank 20 ms
    assert bench.replicas_value(2, 1_000_000, 10, 20.0) == pytest.approx(1000.0)
    assert bench.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]  # one process: identity
