"""The multi-rank host path of bench.py (replicas: one process per GPU, no
data-path collective) on CPU with the gloo backend, world size 2: every rank
gets the slowest rank's time, and the whole-job value counts every rank's
bytes over that time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        slowest = bench.max_over_ranks(0.5 + rank)  # seconds: rank 1 is slower
        gbs = bench.whole_job_gbs(4e9, 10, slowest, world)
        q.put((rank, slowest, gbs))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[1] for g in got] == [1.5, 1.5]
    assert all(g[2] == pytest.approx(2 * 4e9 * 10 / 1.5 / 1e9) for g in got)


def test_single_process_is_its_own_maximum():
    import bench

    assert bench.max_over_ranks(3.25) == 3.25
    assert bench.whole_job_gbs(1e9, 2, 0.5, 1) == pytest.approx(4.0)
