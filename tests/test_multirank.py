"""The N > 1 path of bench.py on CPU: two gloo ranks, each timing its own
replica; the job's time is the maximum over ranks and its value the sum of
all replicas' cell updates over that time."""
import os
import socket

import numpy as np
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


def test_partition_covers_every_request_once_and_balances():
    from mpcns_mercury_b200.distributed import partition

    rng = np.random.default_rng(3)
    work = rng.integers(1, 1000, 101).tolist()
    for world in (1, 2, 3, 8):
        parts = partition(work, world)
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(len(work)))
        loads = [sum(work[q] for q in p) for p in parts]
        assert max(loads) - min(loads) <= max(work)
        assert parts == partition(work, world)  # deterministic


def _serve_rank(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from mpcns_mercury_b200.distributed import aggregate, partition

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # one stream, every rank its own partition; latencies and work made up per request
        work = [10 + (7 * q) % 13 for q in range(40)]
        lat = [0.01 * (q + 1) for q in range(40)]
        mine = partition(work, world)[rank]
        stats = {"cell_updates": sum(work[q] for q in mine), "makespan_s": 1.0 + rank}
        out[rank] = (mine, aggregate(stats, [lat[q] for q in mine]))
        torch.distributed.barrier()
    finally:
        torch.distributed.destroy_process_group()


def test_two_ranks_aggregate_the_latency_percentiles():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_serve_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    mine0, agg0 = res[0]
    mine1, agg1 = res[1]
    assert sorted(mine0 + mine1) == list(range(40)) and not set(mine0) & set(mine1)
    lat = [0.01 * (q + 1) for q in range(40)]
    work = [10 + (7 * q) % 13 for q in range(40)]
    for agg in (agg0, agg1):
        assert agg["requests"] == 40
        assert agg["latency_p50_s"] == pytest.approx(float(np.percentile(lat, 50)))
        assert agg["latency_p99_s"] == pytest.approx(float(np.percentile(lat, 99)))
        assert agg["cell_updates"] == sum(work) and agg["makespan_s"] == 2.0
