"""The N > 1 bench path on CPU: two gloo ranks (127.0.0.1) reduce their step
times to the slowest rank's, and the whole-job throughput counts every
rank's replica."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank
        m = bench.max_over_ranks(ms, dist)
        dist.barrier()
        out.put((rank, m, bench.job_rows_per_s(world, 4, 1000, m)))
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_job_throughput():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [15.0, 15.0]        # both ranks see the slowest rank's time
    assert got[0][2] == pytest.approx(2 * 4 * 1000 / 15e-3)


def test_single_process_needs_no_group():
    import bench

    assert bench.max_over_ranks(3.5, None) == 3.5
