"""The multi-rank path of bench.py on the CPU: two ranks over gloo run the reductions the
bench uses under torchrun (maximum of the per-rank times, sum of throughputs) and the
whole-job value of replicas, with the same call order on every rank."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t_ms = [80.0, 95.0][rank]  # per-rank timed region
        mx = bench.rank_reduce([t_ms], "max", world, "cpu")[0]
        sm = bench.rank_reduce([10.0 + rank, 1.0], "sum", world, "cpu")
        value = bench.replica_value(world, 1000, 18, mx)
        out.put((rank, mx, sm, value))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions_and_replica_value():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(out.get(timeout=10) for _ in range(world))
    for rank, mx, sm, value in res:
        assert mx == 95.0  # the slowest rank's time
        assert sm == [21.0, 2.0]
        assert value == pytest.approx(2 * 1000 * 18 / 0.095)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.rank_reduce([3.0, 4.0], "max", 1, "cpu") == [3.0, 4.0]
    assert bench.replica_value(1, 100, 10, 1000.0) == 1000.0
