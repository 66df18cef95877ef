"""The N > 1 path of bench.py on CPU: replicas only (independent systems per
rank, no collective on the data path), timed as the slowest rank. Two gloo
ranks run the same helpers bench.py uses under torchrun: the max over ranks
of each rank's timed total, and the whole-job throughput over it."""

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        local_ms = 100.0 + 50.0 * rank  # rank 1 is the slower replica
        slowest = bench.max_over_ranks(local_ms, world, "cpu")
        value = bench.replicas_value(1000, 10, slowest, world)
        out.put((rank, slowest, value))
    finally:
        dist.destroy_process_group()


def test_replicas_time_the_slowest_rank():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, value in res:
        assert slowest == pytest.approx(150.0)
        # 2 ranks x 1000 bodies x 10 steps in the slowest rank's 150 ms
        assert value == pytest.approx(2 * 1000 * 10 / 0.150)


def test_single_rank_is_its_own_time():
    import bench

    assert bench.max_over_ranks(42.0, 1, "cpu") == 42.0
    assert bench.replicas_value(1000, 10, 100.0, 1) == pytest.approx(1e5)
