"""The N-GPU bench path is N independent replicas: every rank times its own
step on the device and the reported time is the max over ranks.  This checks
that host logic (bench.max_over_ranks, bench.replica_value) with two gloo
ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 100.0 + 25.0 * rank           # rank 1 is the slowest
        slowest = bench.max_over_ranks(ms, dist, "cpu")
        q.put((rank, slowest, bench.replica_value(world, 1e12, slowest)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, slowest, value in got:
        assert slowest == 125.0
        # two replicas of 1 TFLOP each in 125 ms: 16 TFLOP/s for the job
        assert value == pytest.approx(16.0)


def test_single_process_is_its_own_max():
    import bench
    assert bench.max_over_ranks(42.0, None, "cpu") == 42.0
    assert bench.replica_value(1, 2e12, 1000.0) == pytest.approx(2.0)
