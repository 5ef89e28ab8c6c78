"""Host logic of the multi-GPU path (lps_b200.shard) on CPU: two gloo ranks.

The data path has no collective (instances are independent); these tests
cover the sharding itself, the max-over-ranks job time and the gathering of
per-instance results, with world_size 2 processes on 127.0.0.1.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

from lps_b200.shard import gather_by_instance, job_time_ms, shard


def test_shard_covers_every_instance_once():
    sizes = [31000, 785000, 196321, 196321, 50000, 400000, 120000]
    for world in (1, 2, 3, 4, 8):
        parts = shard(sizes, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        for p in parts:
            assert p == sorted(p)


def test_shard_balances_node_counts():
    sizes = [100] * 8 + [800]
    parts = shard(sizes, 2)
    loads = sorted(sum(sizes[i] for i in p) for p in parts)
    assert loads == [800, 800]
    # more ranks than instances: the extra ranks stay idle
    assert sum(1 for p in shard([5, 6], 4) if not p) == 2


def test_shard_is_deterministic():
    sizes = [7, 7, 7, 7, 3]
    assert shard(sizes, 3) == shard(sizes, 3)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [196321, 196321, 50000, 120000, 400000]
        mine = shard(sizes, world)[rank]
        # each rank's "device time" differs; the job time is the slowest rank's
        t = job_time_ms(10.0 + 5.0 * rank)
        res = gather_by_instance({i: ("rank", rank, i) for i in mine}, len(sizes))
        q.put((rank, mine, t, res))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_and_gather():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (_, mine0, t0, res0), (_, mine1, t1, res1) = out
    assert sorted(mine0 + mine1) == list(range(5)) and not set(mine0) & set(mine1)
    assert t0 == t1 == 15.0
    assert res1 is None
    assert [r[2] for r in res0] == list(range(5))
    assert all(r[1] == (0 if i in mine0 else 1) for i, r in enumerate(res0))


def test_single_process_needs_no_group():
    assert job_time_ms(3.5) == 3.5
    assert gather_by_instance({1: "b", 0: "a"}, 2) == ["a", "b"]


@pytest.mark.gpu
def test_run_shard_matches_one_handle():
    """On one GPU: two ranks' shards, run one after the other, give each
    instance the result of one handle over the whole batch."""
    import numpy as np

    from lps_b200 import gen
    from lps_b200.api import Solver
    from lps_b200.shard import run_shard
    sets = [gen.disc_problem(R=12.0, m=4, nu=0.2, n_steps=40, sigma=3.0),
            gen.disc_problem(R=16.0, m=3, nu=0.4, n_steps=40, sigma=4.0),
            gen.disc_problem(R=10.0, m=5, nu=0.3, n_steps=40, sigma=2.0)]
    parts = {}
    for r in range(2):
        parts.update(run_shard(sets, 40, r, 2, diag_every=10))
    with Solver(sets) as sv:
        sv.step(40, diag_every=10)
        whole = [sv.download(k)["u"] for k in range(len(sets))]
    for i in range(len(sets)):
        np.testing.assert_array_equal(parts[i]["u"], whole[i])
