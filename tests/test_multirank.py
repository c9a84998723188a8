"""Multi-rank plumbing on CPU (gloo, world size 2): column ranges cover every column once,
per-rank seeds differ, and the timing reduction returns the maximum over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from rrtmgp_b200 import shard


def test_column_ranges_partition():
    for total in (1, 7, 8192, 262143):
        for world in (1, 2, 3, 8):
            r = [shard.column_range(total, k, world) for k in range(world)]
            assert r[0][0] == 0 and r[-1][1] == total
            assert all(r[k][1] == r[k + 1][0] for k in range(world - 1))
            lens = [b - a for a, b in r]
            assert max(lens) - min(lens) <= 1
    with pytest.raises(ValueError):
        shard.column_range(10, 2, 2)


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
        ms = 10.0 + 5.0 * rank                        # rank 1 is the slow one
        worst = shard.max_over_ranks(ms, dist)
        rate = shard.weak_scaling_rate(8192, world, 10, worst)
        q.put((rank, worst, rate, shard.rank_seed(42, rank), shard.column_range(100, rank, world)))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_max_and_rate():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(r[1] == 15.0 for r in res)                       # max over ranks
    assert all(abs(r[2] - 2 * 8192 * 10 / 0.015) < 1e-6 for r in res)
    assert res[0][3] != res[1][3]                               # distinct synthetic columns
    assert res[0][4] == (0, 50) and res[1][4] == (50, 100)
