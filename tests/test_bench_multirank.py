"""The replica bookkeeping of bench.py under a 2-rank process group (gloo on
CPU): every rank sees the slowest rank's time, and the whole-job throughput
counts every rank's particles over that time."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    my_ms = 100.0 + 25.0 * rank
    mx = bench.reduce_across_ranks(my_ms, dist, "cpu", "max")
    mn = bench.reduce_across_ranks(my_ms, dist, "cpu", "min")
    val = bench.replica_throughput(world, 1000, 320, mx)
    q.put((rank, mx, mn, val))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_max_time():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, mn, val in res:
        assert mx == 125.0 and mn == 100.0
        assert abs(val - 2 * 1000 * 320 / 0.125) < 1e-6


def test_single_process_no_group():
    import bench
    assert bench.reduce_across_ranks(3.5, None, "cpu") == 3.5
    assert bench.replica_throughput(1, 100, 10, 1.0) == 1e6
