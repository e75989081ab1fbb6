"""The benchmark's multi-GPU form is replicas: every rank ingests its own
seeded cloud and no collective touches the data path. What the ranks share is
the timing: the step time is the maximum over ranks, the points are summed,
and only rank 0 prints. Run here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, world)   # rank 1 is the slower one
    pts = bench.sum_over_ranks(1.0e8, world)               # each rank its own 100M cloud
    bench.barrier(world)
    out.put((rank, ms, pts, pts / (ms / 1e3) / 1e6))
    dist.destroy_process_group()


def test_two_replicas_time_by_the_slowest_rank_and_sum_points():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, pts, value in got:
        assert ms == 15.0 and pts == 2.0e8
        # the whole job's points over the slowest rank's time
        assert value == pytest.approx(2.0e8 / 0.015 / 1e6)
