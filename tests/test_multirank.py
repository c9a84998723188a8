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


def _strong_worker(rank, world, port, q):
    """Rank `rank` of a strong-scaling split: its column range of one 11-column all-sky grid
    through the oracle's LW and SW sequences, gathered on rank 0."""
    import datetime
    import sys
    from pathlib import Path

    import torch.distributed as dist
    repo = Path(__file__).resolve().parent.parent
    sys.path[:0] = [str(repo), str(repo / "rte-rrtmgp-cpp_b200")]
    from oracle import oracle as O
    from rrtmgp_b200 import shard as SH, synthetic as S

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        atm = S.make_atmosphere(11, 9, seed=5, clouds=True)        # every rank builds the same grid
        a, b = SH.column_range(atm["ncol"], rank, world)
        part = SH.slice_columns(atm, a, b)
        lw = O.forward_lw(O.GasOptics(S.make_kdist("lw"), S.ATM_GASES), O.CloudOptics(S.make_cloud_luts("lw")), part)
        sw = O.forward_sw(O.GasOptics(S.make_kdist("sw"), S.ATM_GASES), O.CloudOptics(S.make_cloud_luts("sw")), part)
        res = {"lw_" + k: lw[k] for k in ("flux_up", "flux_dn", "heating_rate")}
        res.update({"sw_" + k: sw[k] for k in ("flux_up", "flux_dn", "flux_dn_dir", "heating_rate")})
        q.put((rank, (a, b), SH.gather_columns(res, dist)))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_strong_split_reproduces_unsharded_run():
    """Strong scaling (one grid's columns split over ranks, results gathered on the host)
    gives exactly the unsharded result: columns are independent."""
    import numpy as np

    from oracle import oracle as O
    from rrtmgp_b200 import synthetic as S
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_strong_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == (0, 6) and res[1][1] == (6, 11) and res[1][2] is None
    got = res[0][2]
    atm = S.make_atmosphere(11, 9, seed=5, clouds=True)
    lw = O.forward_lw(O.GasOptics(S.make_kdist("lw"), S.ATM_GASES), O.CloudOptics(S.make_cloud_luts("lw")), atm)
    sw = O.forward_sw(O.GasOptics(S.make_kdist("sw"), S.ATM_GASES), O.CloudOptics(S.make_cloud_luts("sw")), atm)
    for k in ("flux_up", "flux_dn", "heating_rate"):
        np.testing.assert_array_equal(got["lw_" + k], lw[k])
    for k in ("flux_up", "flux_dn", "flux_dn_dir", "heating_rate"):
        np.testing.assert_array_equal(got["sw_" + k], sw[k])


def test_slice_columns_layouts():
    import numpy as np

    from rrtmgp_b200 import shard as SH, synthetic as S
    atm = S.make_atmosphere(7, 5, seed=1)
    part = SH.slice_columns(atm, 2, 5)
    assert part["ncol"] == 3 and part["play"].shape == (5, 3) and part["plev"].shape == (6, 3)
    assert part["mu0"].shape == (3,) and part["sfc_alb_dir"].shape == (3, 14) and part["emis_sfc"].shape == (3, 16)
    assert part["gases"]["h2o"].shape == (5, 3) and part["gases"]["co2"].shape == (1, 1)
    np.testing.assert_array_equal(part["tlay"], atm["tlay"][:, 2:5])
    with pytest.raises(ValueError):
        SH.slice_columns(atm, 3, 9)
