"""Several ranks (CPU, gloo): the batched clouds dealt to ranks, every point on exactly one
rank, and times reduced to the slowest rank's.  The GPU side of each rank is the 1-GPU
batch path; here each rank builds its forest's plan (the host half)."""
import os
import socket

import numpy as np
import pytest

from fmm_b200.multigpu import max_over_ranks, shard_clouds


def test_shard_clouds_covers_and_balances():
    rng = np.random.default_rng(3)
    sizes = np.exp(rng.uniform(np.log(1e4), np.log(5e5), 256)).astype(np.int64)
    for world in (1, 2, 3, 8):
        parts = shard_clouds(sizes, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [int(sizes[p].sum()) for p in parts]
        # largest-first onto the least loaded: no rank exceeds the mean by more than a cloud
        assert max(loads) - sum(loads) / world <= sizes.max()
        assert shard_clouds(sizes, world) == parts  # every rank computes the same answer
    assert shard_clouds([5, 3], 4) == [[0], [1], [], []]
    with pytest.raises(ValueError):
        shard_clouds([1], 0)


def test_max_over_ranks_without_group():
    assert max_over_ranks(2.5) == 2.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    import fmm_b200 as F

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(11)
        clouds = [rng.uniform(-1, 1, (n, 3)) for n in (900, 3100, 1700, 2500, 600)]
        mine = shard_clouds([len(c) for c in clouds], world)[rank]
        plan = F.FmmBuilder(3).vectors(2).max_points_per_leaf(32).plan_batch([clouds[i] for i in mine])
        info = plan.info()
        import torch

        got = torch.tensor([info["nsources"], len(mine)], dtype=torch.int64)
        dist.all_reduce(got, op=dist.ReduceOp.SUM)
        slowest = max_over_ranks(1.0 + rank)  # a rank-dependent "time"
        out[rank] = (int(got[0]), int(got[1]), slowest, sum(len(clouds[i]) for i in mine))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    total = 900 + 3100 + 1700 + 2500 + 600
    for r in range(2):
        nsrc, ncl, slowest, local = out[r]
        assert nsrc == total and ncl == 5 and slowest == 2.0
    assert out[0][3] + out[1][3] == total and out[0][3] > 0 and out[1][3] > 0


def _failing_rank_main(rank, world, port, out):
    """The batched leg's error path: a rank whose build fails still takes the collective,
    with an infinite time, so that every rank sees the failure and none waits forever."""
    import math

    import torch.distributed as dist

    import fmm_b200 as F

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        cloud = rng.uniform(-1, 1, (800, 3))
        if rank == 1:
            cloud[17, 2] = np.nan  # this rank's build fails on the host
        try:
            F.FmmBuilder(3).max_points_per_leaf(32).plan_batch([cloud])
            t, err = 1.0, ""
        except F.FmmError as e:
            t, err = math.inf, str(e)
        slowest = max_over_ranks(t)
        out[rank] = (slowest, err)
    finally:
        dist.destroy_process_group()


def test_a_failed_rank_is_seen_by_every_rank():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_failing_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert out[0] == (float("inf"), "")
    assert out[1][0] == float("inf") and "non-finite" in out[1][1]
