"""The multi-rank path of bench.py on CPU: two gloo ranks agree on the
slowest rank's time and report the whole job's throughput from it (one
replica per GPU, no data-path collective)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(1.5 + rank, dist, "cpu")      # rank 1 is the slower one
        out.put((rank, t, bench.job_mcells(world, 256 ** 3, 10000, t)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
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
    want = 2 * 256 ** 3 * 10000 / 2.5 / 1e6
    assert [g[1] for g in got] == [2.5, 2.5]
    assert all(g[2] == pytest.approx(want) for g in got)


def test_single_rank_needs_no_process_group():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.job_mcells(1, 100, 10, 1.0) == pytest.approx(1e-3)
