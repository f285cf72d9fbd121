"""Batched sweeps over several GPUs, host side: instances split across ranks
by estimated cost, results gathered on rank 0 in instance order (two gloo
ranks on CPU; the per-rank runner is a stand-in for the GPU sweep)."""
import os
import socket

import numpy as np
import pytest

from openems_b200 import _native as N
from openems_b200 import workloads as W
from openems_b200.sweep import instance_cost, run_sharded, shard_instances

torch = pytest.importorskip("torch")


def test_shards_cover_every_instance_once():
    costs = [instance_cost(s.dims) for s in W.patch_specs(64, seed=4)]
    for world in (1, 2, 3, 4, 8):
        sh = shard_instances(costs, world)
        assert len(sh) == world
        assert sorted(i for s in sh for i in s) == list(range(64))
        assert all(s == sorted(s) for s in sh)
        assert sh == shard_instances(costs, world)  # every rank computes the same split
        loads = [sum(costs[i] for i in s) for s in sh]
        # longest-first greedy: no rank above the mean by more than the largest single instance
        assert max(loads) <= sum(costs) / world + max(costs)
        if world <= 4:
            assert max(loads) / (sum(costs) / world) < 1.1


def test_shard_edge_cases():
    assert shard_instances([], 2) == [[], []]
    assert shard_instances([5.0], 3) == [[0], [], []]
    assert shard_instances([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(N.ConfigError):
        shard_instances([1.0], 0)


def _fake_runner(rank):
    def run_local(indices):
        return {i: {"index": i, "rank": rank, "s11": np.full(3, i + 0.5j)} for i in indices}, 1.0 + rank, \
            100 * len(indices)
    return run_local


def test_single_rank_runs_everything():
    job = run_sharded([3.0, 1.0, 2.0], _fake_runner(0))
    assert [r["index"] for r in job["results"]] == [0, 1, 2]
    assert job["wall_s"] == 1.0 and job["cell_steps"] == 300 and job["shards"] == [[0, 1, 2]]


def test_runner_must_return_its_share():
    with pytest.raises(N.OpenEMSError):
        run_sharded([1.0, 2.0], lambda idx: ({0: {}}, 1.0, 1))
    with pytest.raises(RuntimeError):
        run_sharded([1.0], _failing_runner)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _failing_runner(indices):
    raise RuntimeError("device lost on this rank")


def _rank(rank, world, port, costs, out, fail_rank=-1, own_group=False):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from openems_b200.sweep import run_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # the sweep's command line gathers over a gloo group of its own (beside
    # the NCCL default group); own_group does the same here
    group = dist.new_group(backend="gloo") if own_group else None
    try:
        try:
            job = run_sharded(costs, _failing_runner if rank == fail_rank else _fake_runner(rank), dist, group)
            out.put((rank, job))
        except Exception as e:
            out.put((rank, f"{type(e).__name__}: {e}"))
    finally:
        dist.destroy_process_group()


def _spawn(costs, world, fail_rank=-1, own_group=False):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, costs, q, fail_rank, own_group)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return got


@pytest.mark.parametrize("own_group", (False, True))
def test_failed_rank_is_reported_not_waited_for(own_group):
    """Rank 1's share raises: both ranks return promptly, rank 0 with an
    error naming rank 1, rank 1 with its own exception (over the default
    group, and over a separate gloo group as the command line uses)."""
    got = _spawn([1.0, 2.0, 3.0, 4.0], 2, fail_rank=1, own_group=own_group)
    assert got[0].startswith("OpenEMSError") and "rank 1: RuntimeError: device lost" in got[0]
    assert got[1] == "RuntimeError: device lost on this rank"


def test_two_ranks_gather_on_rank0():
    costs = [instance_cost(s.dims) for s in W.patch_specs(10, seed=4)]
    got = _spawn(costs, 2)
    assert got[1] is None
    job = got[0]
    shards = shard_instances(costs, 2)
    assert job["shards"] == shards
    assert [r["index"] for r in job["results"]] == list(range(10))
    assert all(r["rank"] == (0 if i in shards[0] else 1) for i, r in enumerate(job["results"]))
    assert all(np.array_equal(r["s11"], np.full(3, i + 0.5j)) for i, r in enumerate(job["results"]))
    assert job["wall_s"] == 2.0                      # the slower rank
    assert job["cell_steps"] == 100 * 10
